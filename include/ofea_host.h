/* ofea_host.h - host-side pieces around the GPU hot path, C ABI.
 *
 * These keep OpenFEA's file formats and DOF numbering so the GPU path is a
 * drop-in: the .inp subset the reference reads, set_BCs' free-node numbering
 * and load vector, and the legacy-VTK displacement output.  Pure host code
 * (no GPU needed).  Status codes are those of ofea_gpu.h.
 */
#ifndef OFEA_HOST_H
#define OFEA_HOST_H

#include "ofea_gpu.h" /* status codes, OFEA_API */

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ofea_model ofea_model;

/* ReadInfo::read_ele_node_num / read_geo_mesh / read_load_bcs / read_dis_bcs /
 * read_mat (src/data2cae.cpp:18-53, 77-179, 315-414, 416-446) with the keywords
 * CAE_process::readFile passes ("Set-load", "Cload", "Set-fix",
 * src/cae.cpp:126-130).  Errors (missing file, unknown element type, counts
 * that disagree with the *Nset/*Elset generate lines) return OFEA_ERR_IO
 * instead of exiting. */
OFEA_API int ofea_inp_read(const char *path, ofea_model **out);
OFEA_API void ofea_model_free(ofea_model *m);
OFEA_API int ofea_model_sizes(const ofea_model *m, int *nd, int *ne, int *nfix, int *nload);
/* xyz nd x 3; topo ne x 8 (1-based, as node_topos_); etype (0 C3D4, 1 C3D8);
 * fix (nfix, 1-based, Set-fix order); load_set (nload, 1-based). Any may be NULL. */
OFEA_API int ofea_model_arrays(const ofea_model *m, double *xyz, int *topo, int *etype, int *fix,
                      int *load_set);
/* *Elastic E, nu (has_elastic = 0 when absent: the reference leaves them
 * uninitialised), *Density; Cload DOF (1..3) and value. */
OFEA_API int ofea_model_material(const ofea_model *m, double *E, double *nu, double *density,
                        int *has_elastic);
OFEA_API int ofea_model_cload(const ofea_model *m, int *dof, double *value);

/* The CA change file of the reanalysis (ReadInfo::CA_read_change,
 * src/data2cae.cpp:520-661): every node of the original model with its
 * modified coordinates (*nodes_all), the changed elements (*eles_change:
 * kind 0 deleted, 1 moved, 2 added; etype 0 = C3D4, 1 = C3D8; topo 8 0-based
 * node ids per change, -1 padded), and each node's id in the modified model
 * or -1 (*idref2new).  Sizes are always returned; arrays may be NULL (call
 * once for the sizes, then with arrays of n_nodes*3, n_changes, n_changes,
 * n_changes*8 and n_nodes entries).  OFEA_ERR_IO on a malformed file. */
OFEA_API int ofea_ca_info_read(const char *path, int *n_nodes, int *n_changes, double *xyz, int *kind,
                               int *etype, int *topo, int *node_map);

/* set_BCs::build_free_index (src/set_bc.cpp:20-43): free_map (nd) and the
 * number of free nodes.  Rejects an empty, duplicated or out-of-range fixed
 * set (the reference's loop is undefined there). */
OFEA_API int ofea_build_free_index(int nd, int nfix, const int *fix_ids, int *free_map, int *nfree);
/* set_BCs::build_single_load (src/set_bc.cpp:46-77): f (3*nfree) zeroed, then
 * f[3*free_map[id-1] + dof-1] = value for each load node.  Load nodes that are
 * fixed are skipped (the reference writes out of bounds there). */
OFEA_API int ofea_build_single_load(int nd, const int *free_map, int nload, const int *load_set, int dof,
                           double value, double *f);
/* simulation_post::reset_displacement (src/post_process.cpp:18-39). */
OFEA_API int ofea_full_displacement(int nd, const int *free_map, const double *u, double *u_full);
/* data_process::export_dis_2_vtk (src/data2vtk.cpp:47-264): legacy ASCII VTK,
 * deformed coordinates (scale * u added), cells (C3D8 as VTK type 11 with the
 * reference's node order, C3D4 as type 10), u_x, u_y, u_z, u_magnitude. */
OFEA_API int ofea_write_vtk(const char *path, int nd, const double *xyz, int ne, const int *topo,
                   const int *etype, const double *u_full, double scale);
/* The same, followed by the reference's nodal stress fields S_xx, S_yy,
 * S_zz, S_xy, S_yz, S_xz, S_Mises (src/data2vtk.cpp:211-262) from
 * node_stress [7 x nd] (ofea_stress's node output); NULL writes none. */
OFEA_API int ofea_write_vtk_stress(const char *path, int nd, const double *xyz, int ne, const int *topo,
                                   const int *etype, const double *u_full, double scale,
                                   const double *node_stress);

#ifdef __cplusplus
}
#endif
#endif /* OFEA_HOST_H */
