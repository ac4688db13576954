/*
 * tlfr_oracle.h — CPU restatement of the reference's reconstruction path
 * (TreeGather build + Filterer query, reference src/reconstruction_lib/reconstruction).
 *
 * TEST INFRASTRUCTURE ONLY.  The oracle is the checker for the CUDA path: only
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference legs
 * may load it.  The product library (libtlfr.so) never links or calls it.
 *
 * Parity pinning: tests/test_oracle_vs_reference.py checks this restatement
 * against the reference itself, compiled from its own sources by
 * oracle/build_ref.sh (oracle/_ref/libtlfr_ref*.so), node for node, query by
 * query and pixel by pixel; tests/golden/ holds fixtures generated by the
 * reference build (tests/golden/make_golden.py) for machines without the
 * reference tree.
 */
#ifndef TLFR_ORACLE_H
#define TLFR_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Build the hierarchy (TreeGather::TreeGather, Reconstruction.cpp:43-215).
 * records: W*H*spp*16 floats.  uvt: NULL or the overrideUVT triple.
 * output_spp: 0 = reference default (128, or 1 with uvt).  nthreads: build/query threads. */
int  orc_create(const float* records, int W, int H, int spp, float C0, float C1,
                float aperture, float focus, const float* uvt, int lens_filter, int time_filter,
                int output_spp, int nthreads, void** out, double* build_seconds);

/* reconstructDofMotion (Reconstruction.cpp:221-295).  stats: 16 doubles (Stats, R.hpp:134-147). */
int  orc_reconstruct(void* h, float* rgba, double* seconds, double* stats);

/* Rows [y0,y1) only, into rgba_rows ((y1-y0)*W*4 floats). */
int  orc_reconstruct_rows(void* h, int y0, int y1, float* rgba_rows, double* seconds);

int  orc_tree_info(void* h, int* num_nodes, int* num_samples, int* root, int* spp_pow2,
                   float* coc_adjusted, int* output_spp, int* height);
int  orc_tree_export(void* h, float* nodef, int* nodei, float* samplef, int* sample_ids);
int  orc_output_samples(void* h, float* out5);

/* Grid diagnostics: reprojection grid size and scale, kd-tree node count. */
int  orc_grid_info(void* h, int* grid_w, int* grid_h, float* scale, int* num_initial_nodes,
                   int* num_invalid_bounds);

/* One output sample; trace layout identical to ref_query (ref_driver.cpp). */
int  orc_query(void* h, int x, int y, int i, float* rgba, int* trace, int trace_cap);

void orc_destroy(void* h);
const char* orc_last_error(void);

#ifdef __cplusplus
}
#endif

#endif
