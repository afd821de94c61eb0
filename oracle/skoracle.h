/* skoracle.h -- TEST INFRASTRUCTURE ONLY: the CPU oracle of the photon-packet life cycle.
 *
 * A sequential C restatement of the reference SKIRT 9 algorithm for the hot path
 * (MonteCarloSimulation::performLifeCycle and the grid PathSegmentGenerators). Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg use it, as the checker; the product
 * never links or calls it.
 *
 * The functions mirror the C ABI of include/skgpu.h one to one (same argument meaning), with the
 * prefix or_ instead of skgpu_, so the same host driver runs either. Random numbers come from the
 * same Philox4x32-10 streams keyed by history index, drawn in the reference's order, so the GPU
 * FP64 path and this oracle follow the same histories on identical inputs.
 */
#ifndef SKORACLE_H
#define SKORACLE_H

#include <stdint.h>
#include "../include/skgpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_ctx or_ctx;

int or_create(int device, or_ctx** out);
void or_destroy(or_ctx* ctx);
const char* or_last_error(const or_ctx* ctx);
int or_abi_version(void);
int or_device_count(int32_t* count);

int or_upload_grid_cartesian(or_ctx* ctx, const double* xb, int32_t nxb, const double* yb, int32_t nyb,
                             const double* zb, int32_t nzb);
int or_upload_grid_octree(or_ctx* ctx, int32_t num_nodes, const double* bounds, const int32_t* cell_index,
                          const int32_t* child_begin, const int32_t* child_count, const int32_t* child_index,
                          int32_t num_child_index, const int32_t* nb_begin, const int32_t* nb_index,
                          int32_t num_nb_index, double eps);
int or_upload_grid_adaptive_mesh(or_ctx* ctx, int32_t num_nodes, const double* bounds, const int32_t* cell_index,
                                 const int32_t* child_begin, const int32_t* child_count, const int32_t* child_index,
                                 int32_t num_child_index, double eps);
int or_upload_voronoi_cell_boxes(or_ctx* ctx, int32_t num_cells, const double* boxes);
int or_upload_grid_voronoi(or_ctx* ctx, int32_t num_sites, const double* sites, const int32_t* nb_begin,
                           const int32_t* nb_index, int32_t num_nb_index, const double* extent, double eps);
int or_upload_grid_sphere1d(or_ctx* ctx, int32_t num_borders, const double* radial_borders);
int or_upload_grid_cylinder2d(or_ctx* ctx, int32_t num_radial_borders, const double* radial_borders,
                              int32_t num_z_borders, const double* z_borders);
int or_upload_grid_sphere2d(or_ctx* ctx, int32_t num_radial_borders, const double* radial_borders,
                            int32_t num_polar_borders, const double* polar_borders, const double* polar_cosines);
int or_upload_grid_sphere3d(or_ctx* ctx, int32_t num_radial_borders, const double* radial_borders,
                            int32_t num_polar_borders, const double* polar_borders, const double* polar_cosines,
                            int32_t num_azimuth_borders, const double* azimuth_borders, const double* azimuth_sines,
                            const double* azimuth_cosines, double eps);
int or_upload_grid_cylinder3d(or_ctx* ctx, int32_t num_radial_borders, const double* radial_borders,
                              int32_t num_azimuth_borders, const double* azimuth_borders, const double* azimuth_sines,
                              const double* azimuth_cosines, int32_t num_z_borders, const double* z_borders, double eps,
                              int32_t has_hole);
int or_upload_grid_tetra(or_ctx* ctx, int32_t num_vertices, const double* vertices, int32_t num_tetra,
                         const int32_t* tetra_vertices, const double* face_normals, const int32_t* face_ntetra,
                         const int32_t* face_nface, const double* extent, double eps);
int or_upload_medium(or_ctx* ctx, int32_t num_cells, const double* number_density);
int or_upload_dust_mix(or_ctx* ctx, int32_t num_lambda, const double* lambda_borders, const double* sigma_ext,
                       const double* sigma_sca, const double* asymmpar);
int or_upload_rf_grid(or_ctx* ctx, int32_t num_bins, int32_t num_borders, const double* borders, const int32_t* ellv);
int or_upload_sources(or_ctx* ctx, int32_t num_sources, const skgpu_source* sources, int32_t table_len,
                      const double* table_lambda, const double* table_a, const double* table_b, int32_t radial_len,
                      const double* radial_r, const double* radial_P);
int or_upload_instruments(or_ctx* ctx, int32_t num_instruments, const skgpu_instrument* instruments, int32_t wlg_len,
                          const double* wlg_borders, const int32_t* wlg_ellv);
int or_set_instrument_scattering_levels(or_ctx* ctx, int32_t instrument, int32_t levels);
int or_set_instrument_bands(or_ctx* ctx, int32_t instrument, int32_t num_bands, const int32_t* band_sizes,
                            const double* lambda, const double* transmission, const double* width);
int or_set_instrument_observer(or_ctx* ctx, int32_t instrument, double redshift, double aperture_radius);
int or_set_options(or_ctx* ctx, const skgpu_options* options);
int or_run_primary(or_ctx* ctx, uint64_t first, uint64_t count, uint64_t total_packets);
int or_probe_launch(or_ctx* ctx, uint64_t first, uint64_t count, uint64_t total_packets, double* out);
int or_upload_dust_emission(or_ctx* ctx, int32_t num_rf, const double* rf_sigma_abs, const double* rf_width,
                            const double* rf_cmb, const double* rf_sigma_abs_lum, int32_t num_T, const double* T,
                            const double* planck_abs, int32_t num_em, const double* em_lambda,
                            const double* em_sigma_abs, const double* em_range, int32_t num_cells,
                            const double* cell_volume);
int or_upload_radiation_field(or_ctx* ctx, const double* rf);
int or_prepare_secondary(or_ctx* ctx, const skgpu_secondary_options* options, uint64_t total_packets,
                         double* luminosity);
int or_fetch_dust_emission(or_ctx* ctx, double* luminosity, double* temperature, int32_t* num_points,
                           double* lambda, double* pdf, double* cdf);
int or_run_secondary(or_ctx* ctx, uint64_t first, uint64_t count);
int or_fetch_instrument(or_ctx* ctx, int32_t instrument, double* ifu, double* sed, double* ifu_stats,
                        double* sed_stats);
int or_fetch_instrument_components(or_ctx* ctx, int32_t instrument, double* ifu3, double* sed3);
int or_calibrate_instrument(or_ctx* ctx, int32_t instrument, const double* factors);
int or_fetch_instrument_levels(or_ctx* ctx, int32_t instrument, double* ifu_levels, double* sed_levels);
int or_fetch_radiation_field(or_ctx* ctx, double* rf);
int or_clear_tallies(or_ctx* ctx);
int or_get_counters(or_ctx* ctx, skgpu_counters* out);
int or_last_run_ms(or_ctx* ctx, double* ms);
int or_trace_paths(or_ctx* ctx, int32_t num_rays, const double* rays, int32_t max_segments, int32_t precision,
                   int32_t* count, int32_t* m, double* ds);
int or_optical_depths(or_ctx* ctx, int32_t num_rays, const double* rays, double lambda, int32_t precision,
                      double* tau);

/* C sizes of the ABI records (binding layout test) */
int or_sizeof_source(void);
int or_sizeof_instrument(void);
int or_sizeof_options(void);
int or_sizeof_counters(void);

/* Philox4x32-10 block, exported for known-answer tests */
void or_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

#ifdef __cplusplus
}
#endif

#endif
