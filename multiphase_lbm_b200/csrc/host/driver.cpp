// driver.cpp -- the host driver (include/mlbm_driver.h): command-file parser
// with the reference's token semantics (src/multiphase_lbm.cu:619-745,
// defaults :35-80), geometry and density set-up, and the run loop of
// run_gpu (:565-614) on top of the C ABI of include/mlbm.h.
#include <sys/stat.h>
#include <unistd.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "../../../include/mlbm.h"
#include "../../../include/mlbm_driver.h"
#include "../../../include/mlbm_host.h"
#include "../errors.h"

struct mlbm_driver {
  // lattice size (the reference compiles 400^3 in, include/lbm_model.cuh:4-6)
  int lx = 400, ly = 400, lz = 400;
  int storage = MLBM_STORE_F32;
  int device = 0;
  bool allocated = false;
  std::vector<float> rho;
  std::vector<uint8_t> fluid;
  std::vector<int64_t> solid_number;

  // MultiphaseLBM members and their defaults (src/multiphase_lbm.cu:35-80)
  float res = 1.0f;
  float tau = 1.0f;
  long long step_max = 1000;
  long long step = 0;
  long long vtkPeriod = 10;
  long long statPeriod = 10;
  bool save_vtk_ascii = false;
  std::string result_folder = "./RESULT";
  float rho0 = 0.10f;
  float IniPerturbRate = 1e-3f;
  float G = -1.0f;
  float rhos = 0.0f;
  bool carn_star = false;
  float T_Tc = 0.7f;
  float rhol_spinodal = 0.2726f;
  float rhog_spinodal = 0.0484f;
  bool inject_density = false;
  unsigned inject_type = 0;
  float inject_position = 1.0f;
  unsigned long long rho_inject_period = 100;
  float rho_increment = 0.0f;
  bool read_densities = false;
  std::string densities_filename;
  bool hysteresis = false;
  float max_saturation = 0.98f, min_saturation = 0.04f;
  bool erosion = false;
  float target_density = 0.0f;
  int wanted_num_threads = 4;
  // drainage boundary (absent from the reference)
  int inlet_width = 0, outlet_width = 0;
  float rho_inlet = 0.0f, rho_outlet = 0.0f;

  long long solid_count = 0;
  double packing_density = 0.0;
  mlbm_stats_row last{};
  std::ofstream stat_file;
  mlbm_lattice* lat = nullptr;
};

namespace {

mlbm_status parse_error(const std::string& msg) {
  return mlbm::set_error(MLBM_ERR_PARSE, msg.c_str());
}

// resize_gpu (src/multiphase_lbm.cu:83-157): allocate, initial density
// (from a VTK file when read_densities was given earlier, else the rand()
// perturbation), every node fluid.
mlbm_status resize(mlbm_driver* d) {
  const size_t n = (size_t)d->lx * d->ly * d->lz;
  d->rho.assign(n, 0.f);
  d->fluid.assign(n, 1);
  d->solid_number.assign(n, 0);
  d->allocated = true;
  std::cout << "Setting domain size to: " << d->lx << "x" << d->ly << "x"
            << d->lz << std::endl;
  if (d->read_densities) {
    std::cout << "Reading density data from file: " << d->densities_filename
              << std::endl;
    return mlbm_read_density_vtk(d->densities_filename.c_str(), d->rho.data(),
                                 d->lx, d->ly, d->lz);
  }
  return mlbm_init_density(d->rho.data(), d->lx, d->ly, d->lz, d->rho0,
                           d->IniPerturbRate);
}

mlbm_status ensure_allocated(mlbm_driver* d, const std::string& token) {
  if (d->allocated) return MLBM_OK;
  std::cerr << "token " << token
            << " before resize: allocating the lattice first" << std::endl;
  return resize(d);
}

// read_sample (src/multiphase_lbm.cu:750-806), including the reference's
// reading of the remainder of the size line as the first node (the mask
// comes out shifted by one node, as in the reference).
mlbm_status read_sample(mlbm_driver* d, const std::string& name) {
  std::ifstream file(name);
  if (!file.is_open() || !file.good())
    return mlbm::set_error(MLBM_ERR_IO, ("cannot open sample file " + name).c_str());
  int lxf = 0, lyf = 0, lzf = 0;
  file >> lxf >> lyf >> lzf;
  if (lxf <= 0 || lyf <= 0 || lzf <= 0)
    return parse_error("sample file " + name + ": bad size header");
  const unsigned down = (unsigned)(lxf / d->lx);
  if (down == 0) return parse_error("sample file smaller than the lattice");
  if (mlbm_status st = resize(d)) return st;
  std::vector<uint8_t> ids;
  ids.reserve((size_t)d->lx * d->ly * d->lz);
  std::string line;
  unsigned k = 0;
  while (std::getline(file, line)) {
    const int x = (int)(k / lzf / lyf), y = (int)((k / lzf) % lyf),
              z = (int)(k % lzf);
    if (x % down == 0 && y % down == 0 && z % down == 0) {
      std::istringstream is(line);
      int vid = 0;
      is >> vid;
      ids.push_back(vid != 0);
    }
    ++k;
  }
  const size_t n = (size_t)d->lx * d->ly * d->lz;
  if (ids.size() < n) return parse_error("sample file has too few nodes");
  for (size_t q = 0; q < n; ++q) d->fluid[q] = ids[q] ? 0 : 1;
  d->packing_density = mlbm_packing_density(d->fluid.data(), d->lx, d->ly, d->lz);
  return MLBM_OK;
}

template <typename V>
bool read_value(std::istream& in, V& v) {
  in >> v;
  return !in.fail();
}

}  // namespace

extern "C" {

mlbm_status mlbm_driver_create(mlbm_driver** out) {
  if (!out) return mlbm::set_error(MLBM_ERR_ARG, "null output");
  *out = new (std::nothrow) mlbm_driver();
  return *out ? MLBM_OK : mlbm::set_error(MLBM_ERR_NOMEM, "host allocation");
}

mlbm_status mlbm_driver_destroy(mlbm_driver* d) {
  if (!d) return MLBM_OK;
  if (d->lat) mlbm_lattice_destroy(d->lat);
  delete d;
  return MLBM_OK;
}

mlbm_status mlbm_driver_read(mlbm_driver* d, const char* name) {
  if (!d || !name) return mlbm::set_error(MLBM_ERR_ARG, "null argument");
  std::ifstream file(name);
  if (file.fail())
    return mlbm::set_error(MLBM_ERR_IO,
                           (std::string("cannot open command file ") + name).c_str());
  std::string token;
  file >> token;
  // As in the reference, a token is acted upon only while the stream is
  // good after reading it (a last token not followed by whitespace is not).
  while (file.good()) {
    bool ok = true;
    if (token[0] == '!' || token[0] == '#') {
      std::getline(file, token);
    } else if (token == "result_folder") {
      ok = read_value(file, d->result_folder);
    } else if (token == "num_threads") {
      ok = read_value(file, d->wanted_num_threads);
    } else if (token == "step") {
      ok = read_value(file, d->step);
    } else if (token == "step_max") {
      ok = read_value(file, d->step_max);
    } else if (token == "vtkPeriod") {
      ok = read_value(file, d->vtkPeriod);
      d->save_vtk_ascii = true;
    } else if (token == "vtrPeriod" || token == "tecplotPeriod") {
      long long unused;
      ok = read_value(file, unused);  // parsed, never acted on (as reference)
    } else if (token == "statPeriod") {
      ok = read_value(file, d->statPeriod);
    } else if (token == "rho0") {
      ok = read_value(file, d->rho0);
    } else if (token == "rhos") {
      ok = read_value(file, d->rhos);
    } else if (token == "G") {
      ok = read_value(file, d->G);
    } else if (token == "IniPerturbRate") {
      ok = read_value(file, d->IniPerturbRate);
    } else if (token == "tau") {
      ok = read_value(file, d->tau);
    } else if (token == "resize") {
      if (mlbm_status st = resize(d)) return st;
    } else if (token == "read_sample") {
      std::string f;
      ok = read_value(file, f);
      if (ok) {
        std::cout << "Reading node ids from: " << f << std::endl;
        if (mlbm_status st = read_sample(d, f)) return st;
      }
    } else if (token == "place_sphere") {
      float x, y, z, R;
      ok = read_value(file, x) && read_value(file, y) && read_value(file, z) &&
           read_value(file, R);
      if (ok) {
        if (mlbm_status st = ensure_allocated(d, token)) return st;
        // the grain counter is not advanced (src/multiphase_lbm.cu:669-674)
        if (mlbm_status st = mlbm_place_sphere(d->fluid.data(), d->solid_number.data(),
                                               d->lx, d->ly, d->lz, x, y, z, R,
                                               d->solid_count))
          return st;
        std::cout << "Placing sphere with radius " << R << " at (" << x << ", "
                  << y << ", " << z << ")" << std::endl;
      }
    } else if (token == "generate_solids") {
      int num;
      float rmin, rmax, x0, x1, y0, y1, z0, z1;
      ok = read_value(file, num) && read_value(file, rmin) &&
           read_value(file, rmax) && read_value(file, x0) &&
           read_value(file, x1) && read_value(file, y0) &&
           read_value(file, y1) && read_value(file, z0) && read_value(file, z1);
      if (ok) {
        if (mlbm_status st = ensure_allocated(d, token)) return st;
        int64_t cnt = d->solid_count;
        if (mlbm_status st = mlbm_generate_solids(
                d->fluid.data(), d->solid_number.data(), d->lx, d->ly, d->lz,
                num, rmin, rmax, x0, x1, y0, y1, z0, z1, &cnt))
          return st;
        d->solid_count = cnt;
      }
    } else if (token == "resolution") {
      ok = read_value(file, d->res);
    } else if (token == "read_positions") {
      std::string f;
      ok = read_value(file, f);
      if (ok) {
        if (mlbm_status st = ensure_allocated(d, token)) return st;
        std::cout << "Reading grain positions and radii from: " << f
                  << "\nwith resolution of: " << d->res << std::endl;
        int64_t cnt = d->solid_count;
        if (mlbm_status st = mlbm_read_positions(f.c_str(), d->res, d->fluid.data(),
                                                 d->solid_number.data(), d->lx,
                                                 d->ly, d->lz, &cnt))
          return st;
        d->solid_count = cnt;
        std::cout << "number of grain = " << d->solid_count << std::endl;
        d->packing_density =
            mlbm_packing_density(d->fluid.data(), d->lx, d->ly, d->lz);
        std::cout << "Packing density: " << (float)d->packing_density << std::endl;
      }
    } else if (token == "rho_inject_period") {
      ok = read_value(file, d->rho_inject_period);
    } else if (token == "rho_increment") {
      d->inject_density = true;
      ok = read_value(file, d->rho_increment);
    } else if (token == "inject_type") {
      ok = read_value(file, d->inject_type);
    } else if (token == "inject_position") {
      ok = read_value(file, d->inject_position);
    } else if (token == "carn_star") {
      d->carn_star = true;
    } else if (token == "T_Tc") {
      ok = read_value(file, d->T_Tc);
    } else if (token == "rhol_spinodal") {
      ok = read_value(file, d->rhol_spinodal);
    } else if (token == "rhog_spinodal") {
      ok = read_value(file, d->rhog_spinodal);
    } else if (token == "read_densities") {
      ok = read_value(file, d->densities_filename);
      d->read_densities = true;
    } else if (token == "max_saturation") {
      ok = read_value(file, d->max_saturation);
      d->hysteresis = true;
    } else if (token == "min_saturation") {
      ok = read_value(file, d->min_saturation);
    } else if (token == "target_density") {
      ok = read_value(file, d->target_density);
      d->erosion = true;
    // ---- tokens the reference does not parse ----
    } else if (token == "lx" || token == "lxSample") {
      ok = read_value(file, d->lx);
    } else if (token == "ly" || token == "lySample") {
      ok = read_value(file, d->ly);
    } else if (token == "lz" || token == "lzSample") {
      ok = read_value(file, d->lz);
    } else if (token == "storage") {
      std::string s;
      ok = read_value(file, s);
      if (s == "f32") d->storage = MLBM_STORE_F32;
      else if (s == "f16") d->storage = MLBM_STORE_F16;
      else if (s == "f64") d->storage = MLBM_STORE_F64;
      else return parse_error("storage must be f32, f16 or f64");
    } else if (token == "device") {
      ok = read_value(file, d->device);
    } else if (token == "inlet_width") {
      ok = read_value(file, d->inlet_width);
    } else if (token == "outlet_width") {
      ok = read_value(file, d->outlet_width);
    } else if (token == "rho_inlet") {
      ok = read_value(file, d->rho_inlet);
    } else if (token == "rho_outlet") {
      ok = read_value(file, d->rho_outlet);
    } else if (token == "G_ads") {
      float gads;
      ok = read_value(file, gads);
      if (ok) {
        // G_ads = G psi(rhos)  =>  rhos = -ln(1 - G_ads / G)
        if (d->G == 0.f || gads / d->G >= 1.f)
          return parse_error("G_ads needs a nonzero G with G_ads/G < 1");
        d->rhos = (float)(-std::log(1.0 - (double)gads / (double)d->G));
      }
    } else if (token == "generate_packing") {
      float rmin, rmax;
      double porosity;
      unsigned long long seed;
      ok = read_value(file, rmin) && read_value(file, rmax) &&
           read_value(file, porosity) && read_value(file, seed);
      if (ok) {
        if (mlbm_status st = ensure_allocated(d, token)) return st;
        std::vector<float> xyzr((size_t)d->lx * d->ly * d->lz / 4 + 16);
        int64_t cnt = 0;
        double por = 0;
        if (mlbm_status st = mlbm_generate_packing(
                d->lx, d->ly, d->lz, rmin, rmax, porosity, seed,
                (int64_t)(xyzr.size() / 4), d->fluid.data(), xyzr.data(), &cnt,
                &por))
          return st;
        for (int64_t s = 0; s < cnt; ++s) {
          d->solid_count += 1;
          mlbm_place_sphere(d->fluid.data(), d->solid_number.data(), d->lx,
                            d->ly, d->lz, xyzr[4 * s], xyzr[4 * s + 1],
                            xyzr[4 * s + 2], xyzr[4 * s + 3], d->solid_count);
        }
        d->packing_density = 1.0 - por;
        std::cout << "Generated " << cnt << " grains, porosity " << por
                  << std::endl;
      }
    } else {
      std::cerr << "The token " << token << "is undefined." << std::endl;
    }
    if (!ok) return parse_error("missing or malformed value after token " + token);
    file >> token;
  }
  std::cout << "rho0: " << d->rho0 << std::endl;
  std::cout << "perturbation rate: " << d->IniPerturbRate << std::endl;
  std::cout << "rhos: " << d->rhos << std::endl;
  if (d->carn_star)
    std::cout << "Using Carnahan-Starling EOS with T/Tc = " << d->T_Tc
              << ", rhol* = " << d->rhol_spinodal
              << " and rhog* = " << d->rhog_spinodal << std::endl;
  else
    std::cout << "Using Shan-Chen EOS with G = " << d->G << std::endl;
  if (d->erosion)
    std::cerr << "target_density: erosion is not supported; geometry unchanged"
              << std::endl;
  return MLBM_OK;
}

mlbm_status mlbm_driver_init(mlbm_driver* d) {
  if (!d) return mlbm::set_error(MLBM_ERR_ARG, "null driver");
  if (access(d->result_folder.c_str(), F_OK))
    mkdir(d->result_folder.c_str(), S_IRUSR | S_IWUSR | S_IXUSR | S_IRGRP |
                                        S_IXGRP | S_IROTH | S_IXOTH);
  std::cout << "Resulting files will be saved in " << d->result_folder
            << std::endl;
  d->stat_file.open(d->result_folder + "/Stats.txt");
  if (!d->stat_file)
    return mlbm::set_error(MLBM_ERR_IO, "cannot create Stats.txt");
  d->stat_file << "step\tmin_rho\tmax_rho\tmin_p\tmax_p\t"
                  "avg_liq_press\tavg_vap_press\t"
                  "suction\tSr\tavg_liq_rho\tavg_vap_rho\t"
                  "liq_cluster_count\tcluster_order\twet_coord_num\tgas_cluster_"
                  "count\tliquid_solid_boundary\tliquid_vapor_boundary\tcluster_radius"
               << std::endl;
  return MLBM_OK;
}

mlbm_status mlbm_driver_params(const mlbm_driver* d, mlbm_params* p) {
  if (!d || !p) return mlbm::set_error(MLBM_ERR_ARG, "null argument");
  std::memset(p, 0, sizeof *p);
  p->tau = d->tau;
  p->G = d->G;
  p->T_Tc = d->T_Tc;
  p->rhol_spinodal = d->rhol_spinodal;
  p->rhog_spinodal = d->rhog_spinodal;
  p->rho_increment = d->rho_increment;
  p->rhos = d->rhos;
  p->inject_position = d->inject_position;
  p->carn_star = d->carn_star;
  p->inject_density = d->inject_density;
  p->rho_inject_period = d->rho_inject_period;
  p->stat_period = (uint64_t)d->statPeriod;
  p->inlet_width = d->inlet_width;
  p->outlet_width = d->outlet_width;
  p->rho_inlet = d->rho_inlet;
  p->rho_outlet = d->rho_outlet;
  p->rho_shift = 1.0f;
  return MLBM_OK;
}

}  // extern "C"

// Statistics of the current state: phase averages on the device, then the
// cluster columns of the downloaded density on the device as well
// (calc_cluster + write_stats, src/multiphase_lbm.cu:225-562, 1057-1083).  Averages the reference leaves untouched when a
// phase is empty keep their previous values.
mlbm_status driver_stats(mlbm_driver* d, std::vector<float>& rho_host) {
  mlbm_stats s;
  if (mlbm_status st = mlbm_phase_stats(d->lat, &s)) return st;
  mlbm_stats_row& r = d->last;
  r.step = d->step;
  r.min_rho = (float)s.min_rho;
  r.max_rho = (float)s.max_rho;
  r.min_p = (float)s.min_p;
  r.max_p = (float)s.max_p;
  if (s.n_liquid) {
    r.avg_liq_press = (float)s.avg_p_liquid;
    r.avg_liq_rho = (float)s.avg_rho_liquid;
  }
  if (s.n_vapour) {
    r.avg_vap_press = (float)s.avg_p_vapour;
    r.avg_vap_rho = (float)s.avg_rho_vapour;
  }
  r.suction = (float)(r.avg_vap_press - r.avg_liq_press);
  r.saturation = (float)((float)s.n_liquid / (float)s.n_fluid);
  if (mlbm_status st = mlbm_download_field(d->lat, MLBM_FIELD_RHO, MLBM_DTYPE_F32,
                                           rho_host.data()))
    return st;
  return mlbm_cluster_stats_gpu(rho_host.data(), d->fluid.data(),
                                d->solid_number.data(), d->lx, d->ly, d->lz,
                                d->rhol_spinodal, d->rhog_spinodal,
                                d->solid_count, d->device, nullptr, nullptr, &r);
}

void write_stats_row(std::ofstream& f, const mlbm_stats_row& r) {
  // the reference streams `real` (float) values with default formatting
  f << r.step << "\t" << (float)r.min_rho << "\t" << (float)r.max_rho << "\t"
    << (float)r.min_p << "\t" << (float)r.max_p << "\t" << (float)r.avg_liq_press
    << "\t" << (float)r.avg_vap_press << "\t" << (float)r.suction << "\t"
    << (float)r.saturation << "\t" << (float)r.avg_liq_rho << "\t"
    << (float)r.avg_vap_rho << "\t" << r.liq_cluster_count << "\t"
    << (float)r.cluster_order << "\t" << (float)r.wet_coord_num << "\t"
    << r.gas_cluster_count << "\t" << (float)r.liquid_solid_boundary << "\t"
    << (float)r.liquid_vapor_boundary << "\t" << (float)r.cluster_radius
    << std::endl
    << std::flush;
}

extern "C" mlbm_status mlbm_driver_run(mlbm_driver* d, int32_t quiet) {
  if (!d) return mlbm::set_error(MLBM_ERR_ARG, "null driver");
  if (!d->allocated) return mlbm::set_error(MLBM_ERR_STATE, "no lattice: missing resize");
  if (d->statPeriod <= 0) return mlbm::set_error(MLBM_ERR_ARG, "statPeriod must be > 0");
  if (d->lat) {
    mlbm_lattice_destroy(d->lat);
    d->lat = nullptr;
  }
  if (mlbm_status st = mlbm_lattice_create(d->lx, d->ly, d->lz, d->storage,
                                           d->device, &d->lat))
    return st;
  mlbm_params p;
  mlbm_driver_params(d, &p);
  if (mlbm_status st = mlbm_set_params(d->lat, &p)) return st;
  if (mlbm_status st = mlbm_upload_fluid_mask(d->lat, d->fluid.data())) return st;
  if (mlbm_status st = mlbm_upload_rho(d->lat, d->rho.data())) return st;
  if (mlbm_status st = mlbm_initialize(d->lat)) return st;
  std::vector<float> rho_host(d->rho.size());
  const int reverse = 1;  // fixed in the reference (src/multiphase_lbm.cu:573)
  long long num_vtk = 0;
  while (d->step < d->step_max) {
    // advance to the next statistics step (inclusive) in one call
    long long next = (d->step / d->statPeriod + (d->step % d->statPeriod ? 1 : 0)) *
                     d->statPeriod;
    if (next < d->step) next = d->step;
    const long long last = std::min(next, d->step_max - 1);
    const int32_t n = (int32_t)(last - d->step + 1);
    if (mlbm_status st = mlbm_iterate(d->lat, d->step, n, reverse,
                                      d->inject_type, 0))
      return st;
    d->step = last;
    if (d->step % d->statPeriod == 0) {
      if (mlbm_status st = driver_stats(d, rho_host)) return st;
      if (!quiet)
        std::printf("saturation=%f, aLp=%f,aVp=%f, step=%lld\n",
                    (float)d->last.saturation, (float)d->last.avg_liq_press,
                    (float)d->last.avg_vap_press, d->step);
      if (d->stat_file.is_open()) write_stats_row(d->stat_file, d->last);
      if (d->save_vtk_ascii && d->vtkPeriod > 0 && d->step % d->vtkPeriod == 0) {
        if (!quiet)
          std::cout << "Saving vtk ascii file number " << num_vtk << std::endl;
        if (mlbm_status st = mlbm_driver_write_vtk(d, num_vtk)) return st;
        ++num_vtk;
      }
    }
    d->step += 1;
  }
  return mlbm_synchronize(d->lat);
}

extern "C" {

mlbm_status mlbm_driver_dims(const mlbm_driver* d, int32_t* dims) {
  if (!d || !dims) return mlbm::set_error(MLBM_ERR_ARG, "null argument");
  dims[0] = d->lx;
  dims[1] = d->ly;
  dims[2] = d->lz;
  return MLBM_OK;
}

mlbm_status mlbm_driver_arrays(mlbm_driver* d, float** rho, uint8_t** fluid,
                               int64_t** sn) {
  if (!d) return mlbm::set_error(MLBM_ERR_ARG, "null driver");
  if (!d->allocated) return mlbm::set_error(MLBM_ERR_STATE, "no lattice allocated");
  if (rho) *rho = d->rho.data();
  if (fluid) *fluid = d->fluid.data();
  if (sn) *sn = d->solid_number.data();
  return MLBM_OK;
}

mlbm_status mlbm_driver_last_stats(const mlbm_driver* d, mlbm_stats_row* row) {
  if (!d || !row) return mlbm::set_error(MLBM_ERR_ARG, "null argument");
  *row = d->last;
  return MLBM_OK;
}

mlbm_status mlbm_driver_info(const mlbm_driver* d, int64_t* step,
                             int64_t* step_max, int64_t* stat_period,
                             int64_t* vtk_period, int64_t* solid_count,
                             double* packing_density, int32_t* storage) {
  if (!d) return mlbm::set_error(MLBM_ERR_ARG, "null driver");
  if (step) *step = d->step;
  if (step_max) *step_max = d->step_max;
  if (stat_period) *stat_period = d->statPeriod;
  if (vtk_period) *vtk_period = d->save_vtk_ascii ? d->vtkPeriod : -1;
  if (solid_count) *solid_count = d->solid_count;
  if (packing_density) *packing_density = d->packing_density;
  if (storage) *storage = d->storage;
  return MLBM_OK;
}

mlbm_lattice* mlbm_driver_lattice(mlbm_driver* d) { return d ? d->lat : nullptr; }

}  // extern "C"

std::string driver_result_folder(const mlbm_driver* d) { return d->result_folder; }
int driver_device(const mlbm_driver* d) { return d->device; }
