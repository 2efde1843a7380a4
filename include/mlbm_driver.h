/*
 * mlbm_driver.h -- the host driver of libmlbm behind a C ABI: the reference's
 * MultiphaseLBM run surface (include/multiphase_lbm.h:26-218 of
 * Amber1995/multiphase_LBM) -- read a command file, build the geometry and
 * initial density, run the time loop on the GPU, write Stats.txt and VTK
 * files -- with the same command-file format.
 *
 *   reference                                   this ABI
 *   MultiphaseLBM::read_data(file)  :619-745    mlbm_driver_read
 *   MultiphaseLBM::init()           :930-944    mlbm_driver_init
 *   MultiphaseLBM::run_gpu()        :565-614    mlbm_driver_run
 *   calc_cluster + write_stats      :225-562, 1057-1083  (inside run)
 *   write_vtk_ascii                 :948-1054   mlbm_driver_write_vtk
 *   main(argc, argv)                src/main.cc:4-17     the `mlbm` program
 *
 * Command-file tokens: every token of the reference parser, with its
 * semantics and defaults, plus tokens for what the reference fixes at compile
 * time or does not have:
 *   lx N / ly N / lz N (aliases lxSample/lySample/lzSample): lattice size
 *     (default 400 each, the reference's compiled size); must precede resize.
 *   storage f32|f16|f64: population storage (default f32).
 *   inlet_width N, rho_inlet R, outlet_width N, rho_outlet R: drainage slabs.
 *   G_ads A: wall adhesion; sets rhos = -ln(1 - A/G) (needs G first).
 *   generate_packing rmin rmax porosity seed: seeded sphere packing.
 *   device N: CUDA device.
 * target_density (erosion) is parsed but not applied (a warning is printed).
 */
#ifndef MLBM_DRIVER_H_
#define MLBM_DRIVER_H_

#include <stdint.h>

#include "mlbm.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mlbm_driver mlbm_driver;

/* One row of Stats.txt (src/multiphase_lbm.cu:937-943, 1073-1082). */
typedef struct mlbm_stats_row {
  int64_t step;
  double min_rho, max_rho, min_p, max_p;
  double avg_liq_press, avg_vap_press, suction, saturation;
  double avg_liq_rho, avg_vap_rho;
  int64_t liq_cluster_count;
  double cluster_order, wet_coord_num;
  int64_t gas_cluster_count;
  double liquid_solid_boundary, liquid_vapor_boundary, cluster_radius;
} mlbm_stats_row;

mlbm_status mlbm_driver_create(mlbm_driver** out);
mlbm_status mlbm_driver_destroy(mlbm_driver* d);
/* Parse a command file and apply its actions (geometry, density). */
mlbm_status mlbm_driver_read(mlbm_driver* d, const char* command_file);
/* Create the result folder and Stats.txt with its header. */
mlbm_status mlbm_driver_init(mlbm_driver* d);
/* Run steps [step, step_max) with statistics every statPeriod steps and VTK
 * output every vtkPeriod steps (when vtkPeriod was given).  quiet = 0 prints
 * the reference's progress lines. */
mlbm_status mlbm_driver_run(mlbm_driver* d, int32_t quiet);
/* Write result%06d.vtk of the current state. */
mlbm_status mlbm_driver_write_vtk(mlbm_driver* d, int64_t num);

/* Introspection (sizes, the host arrays the driver holds, last stats). */
mlbm_status mlbm_driver_dims(const mlbm_driver* d, int32_t* dims);
/* Host arrays in the reference layout [x][y][z]: rho (float), is_fluid
 * (uint8), solid_number (int64).  Valid until the driver is destroyed. */
mlbm_status mlbm_driver_arrays(mlbm_driver* d, float** rho, uint8_t** fluid,
                               int64_t** solid_number);
mlbm_status mlbm_driver_params(const mlbm_driver* d, mlbm_params* p);
mlbm_status mlbm_driver_last_stats(const mlbm_driver* d, mlbm_stats_row* row);
/* Info: step, step_max, statPeriod, vtkPeriod (-1 if unset), solid_count,
 * packing_density, storage. */
mlbm_status mlbm_driver_info(const mlbm_driver* d, int64_t* step,
                             int64_t* step_max, int64_t* stat_period,
                             int64_t* vtk_period, int64_t* solid_count,
                             double* packing_density, int32_t* storage);
/* The lattice the driver runs (NULL before mlbm_driver_run). */
mlbm_lattice* mlbm_driver_lattice(mlbm_driver* d);

/* Cluster statistics of calc_cluster (src/multiphase_lbm.cu:225-562) on host
 * arrays in the reference layout, without recursion.  liq/gas labels
 * (optional, int64 [x][y][z]) receive the cluster numbers.  out receives the
 * cluster columns and boundary ratios of a Stats.txt row (the other fields
 * are left untouched). */
mlbm_status mlbm_cluster_stats(const float* rho, const uint8_t* is_fluid,
                               const int64_t* solid_number, int32_t nx,
                               int32_t ny, int32_t nz, float rhol_spinodal,
                               float rhog_spinodal, int64_t solid_count,
                               int64_t* liq_labels, int64_t* gas_labels,
                               mlbm_stats_row* out);

/* The same statistics computed on GPU `device` (connected components by a
 * lock-free union-find rooted at the first node of the reference's scan,
 * cluster-solid contacts sorted on the device).  Same arguments, results and
 * labels as mlbm_cluster_stats; the host arrays are copied in, the labels
 * (optional) copied out.  Replaces the host-side calc_cluster
 * (src/multiphase_lbm.cu:225-562) for large lattices (< 2^31 nodes). */
mlbm_status mlbm_cluster_stats_gpu(const float* rho, const uint8_t* is_fluid,
                                   const int64_t* solid_number, int32_t nx,
                                   int32_t ny, int32_t nz, float rhol_spinodal,
                                   float rhog_spinodal, int64_t solid_count,
                                   int32_t device, int64_t* liq_labels,
                                   int64_t* gas_labels, mlbm_stats_row* out);

#ifdef __cplusplus
}
#endif

#endif /* MLBM_DRIVER_H_ */
