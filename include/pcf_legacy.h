/*
 * pcf_legacy.h -- the reference's C++ host entry points, same names and
 * signatures (cuda/pcf2iso.cuh:11, pcf2ani.cuh:5, pcf2isoBPC.cuh:11,166,
 * pcf2aniBPC.cuh:5, pcf3iso.cuh:10, pcf3isoBPC.cuh:10,177, pcf3ani.cuh:10,
 * pcf3aniBPC.cuh:10), implemented on libpcf.so.
 *
 * Arguments mean what they mean there: device arrays of cell descriptors
 * (DNode) and cell-ordered points (PointW3D) as cuda/main.cu:281-329 builds
 * them, the random catalogs packed at offsets i*np with their cell
 * descriptors at acum_nonzero_Rnodes[i]; histo_names[0] the data name and
 * histo_names[i+1] the random names.  Each writes the reference's result
 * files to ../results/ (save_histogram1D/2D/3D, cuda/create_grid.cuh:141-266)
 * and prints the elapsed time.  Unlike the reference they report failures
 * by printing a message and returning instead of exit(-1).
 *
 * Include after the reference's create_grid.cuh with
 * PCF_LEGACY_HAVE_REFERENCE_TYPES defined, or alone to get the layouts.
 */
#ifndef PCF_LEGACY_H
#define PCF_LEGACY_H

#include <string>

#ifndef PCF_LEGACY_HAVE_REFERENCE_TYPES
struct Point3D { float x, y, z; };                 // create_grid.cuh:8
struct PointW3D { float x, y, z, w; };             // create_grid.cuh:15
struct DNode { Point3D nodepos; int len; int start; int end; };  // create_grid.cuh:28
#endif

void pcf_2iso(std::string *histo_names, DNode *dnodeD, PointW3D *d_ordered_pointsD,
              int nonzero_Dnodes, DNode *dnodeR, PointW3D *d_ordered_pointsR, int *nonzero_Rnodes,
              int *acum_nonzero_Rnodes, int n_randfiles, int bn, float size_node, float dmax);
void pcf_2ani(std::string *histo_names, DNode *dnodeD, PointW3D *d_ordered_pointsD,
              int nonzero_Dnodes, DNode *dnodeR, PointW3D *d_ordered_pointsR, int *nonzero_Rnodes,
              int *acum_nonzero_Rnodes, int n_randfiles, int bn, float size_node, float dmax);
void pcf_2iso_BPC(std::string *histo_names, DNode *dnodeD, PointW3D *d_ordered_pointsD,
                  int nonzero_Dnodes, DNode *dnodeR, PointW3D *d_ordered_pointsR,
                  int *nonzero_Rnodes, int *acum_nonzero_Rnodes, int n_randfiles, int bn,
                  float size_node, float size_box, float dmax);
void pcf_2iso_BPCanalytic(std::string histo_names, DNode *dnodeD, PointW3D *d_ordered_pointsD,
                          int nonzero_Dnodes, int bn, int np, float size_node, float size_box,
                          float dmax);
void pcf_2aniBPC(std::string *histo_names, DNode *dnodeD, PointW3D *d_ordered_pointsD,
                 int nonzero_Dnodes, DNode *dnodeR, PointW3D *d_ordered_pointsR,
                 int *nonzero_Rnodes, int *acum_nonzero_Rnodes, int n_randfiles, int bn,
                 float size_node, float size_box, float dmax);
void pcf_3iso(std::string *histo_names, DNode *dnodeD, PointW3D *d_ordered_pointsD,
              int nonzero_Dnodes, DNode *dnodeR, PointW3D *d_ordered_pointsR, int *nonzero_Rnodes,
              int *acum_nonzero_Rnodes, int n_randfiles, int bn, float size_node, float dmax);
void pcf_3isoBPC(std::string *histo_names, DNode *dnodeD, PointW3D *d_ordered_pointsD,
                 int nonzero_Dnodes, DNode *dnodeR, PointW3D *d_ordered_pointsR,
                 int *nonzero_Rnodes, int *acum_nonzero_Rnodes, int n_randfiles, int bn,
                 float size_node, float size_box, float dmax);
void pcf_3isoBPC_analytic(std::string data_name, DNode *dnodeD, PointW3D *d_ordered_pointsD,
                          int nonzero_Dnodes, int bn, int np, float size_node, float size_box,
                          float dmax);
void pcf_3ani(std::string *histo_names, DNode *dnodeD, PointW3D *d_ordered_pointsD,
              int nonzero_Dnodes, DNode *dnodeR, PointW3D *d_ordered_pointsR, int *nonzero_Rnodes,
              int *acum_nonzero_Rnodes, int n_randfiles, int bn, float size_node, float dmax);
void pcf_3aniBPC(std::string *histo_names, DNode *dnodeD, PointW3D *d_ordered_pointsD,
                 int nonzero_Dnodes, DNode *dnodeR, PointW3D *d_ordered_pointsR,
                 int *nonzero_Rnodes, int *acum_nonzero_Rnodes, int n_randfiles, int bn,
                 float size_node, float size_box, float dmax);

#endif
