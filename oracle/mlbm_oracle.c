/*
 * mlbm_oracle.c -- TEST INFRASTRUCTURE ONLY (the oracle).  Never linked into
 * or called by the product; only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py use it, to verify results.
 *
 * A plain-C restatement, with runtime lattice sizes, of the reference's D3Q19
 * single-component Shan-Chen time step (Amber1995/multiphase_LBM):
 *
 *   step n:  pull streaming + halfway bounce-back
 *              (include/iteration_device.cuh:252-271,
 *               include/iteration_kernel.cuh:51-62, 65-118)
 *            density + injection, pressure, psi for every fluid node
 *              (include/iteration_device.cuh:40-63)
 *            Shan-Chen force from psi of the 18 neighbours
 *              (include/iteration_device.cuh:69-152)
 *            velocity shift u = (sum f e + tau F) / rho, BGK
 *              (include/iteration_device.cuh:162-206)
 *            swap lattices (include/iteration_kernel.cuh:44-48)
 *   init:    f_i = t_i rho everywhere; solids get rho = rhos, psi(rhos), F = 0
 *              (include/iteration_kernel.cuh:9-29)
 *
 * Arithmetic follows the reference expression by expression (float storage,
 * double-promoted literals where the reference has them) so that, compiled
 * with -ffp-contract=off like the reference build in oracle/_ref, the FP32
 * build reproduces the reference bit for bit.  Built with -DMLBMO_F64 every
 * quantity is double: the FP64 oracle of the same update.
 *
 * The collision runs as two sweeps (all densities, then all forces and
 * relaxations): the race-free order.  The reference GPU kernel
 * (include/iteration_kernel.cuh:32-41) reads neighbour psi while other
 * threads of the same launch overwrite it.
 *
 * Build-defined drainage boundary (absent from the reference): fluid nodes
 * with x < inlet_width are held at rho_inlet, with x >= lx - outlet_width at
 * rho_outlet: their rho and psi are fixed and their post-collision
 * populations are the rest equilibrium t_i * rho.
 *
 * Layout is the reference's: scalars [x][y][z] (z fastest), populations
 * [x][y][z][19], force [x][y][z][3].
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef MLBMO_F64
typedef double real;
#define EXPR(x) exp(x)
#define SQRTR(x) sqrt(x)
#define SYM(name) mlbmo64_##name
#else
typedef float real;
#define EXPR(x) expf(x)
#define SQRTR(x) sqrt(x)
#define SYM(name) mlbmo32_##name
#endif

enum { Q = 19, HALF = 9 };

/* D3Q19 tables, include/lbm_model.cuh:35-54 (the direction order and
 * weights are the reference's; opposite(i) = i +- 9, :24). */
static const int EX[Q] = {0, -1, 0, 0, -1, -1, -1, -1, 0, 0,
                          1, 0, 0, 1, 1, 1, 1, 0, 0};
static const int EY[Q] = {0, 0, -1, 0, -1, 1, 0, 0, -1, -1,
                          0, 1, 0, 1, -1, 0, 0, 1, 1};
static const int EZ[Q] = {0, 0, 0, -1, 0, 0, -1, 1, -1, 1,
                          0, 0, 1, 0, 0, 1, -1, 1, -1};

typedef struct {
  float tau, G, T_Tc, rhol_spinodal, rhog_spinodal, rho_increment, rhos,
      inject_position;
  int32_t carn_star, inject_density;
  uint64_t rho_inject_period, stat_period;
  int32_t inlet_width, outlet_width;
  float rho_inlet, rho_outlet;
} mlbmo_params;

typedef struct {
  int lx, ly, lz;
  size_t n;
  mlbmo_params p;
  real t[Q];
  real *rho, *psi, *pressure, *force, *vel, *fa, *fb; /* fa = collision_f */
  uint8_t* fluid;
} mlbmo;

static inline size_t idx(const mlbmo* o, int x, int y, int z) {
  return ((size_t)x * o->ly + y) * o->lz + z;
}

static inline int wrap(int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); }

/* dPress, include/iteration_device.cuh:7-27 */
static real press(const mlbmo* o, real rho) {
  if (o->p.carn_star) {
    real a = 1.0, b = 4.0, R = 1.0, Tc = 0.0943;
    real T = (real)o->p.T_Tc * Tc;
    real eta = b * rho / 4.0;
    real eta2 = eta * eta, eta3 = eta2 * eta, rho2 = rho * rho;
    real ome = (1.0 - eta);
    real ome3 = ome * ome * ome;
    return rho * R * T * (1 + eta + eta2 - eta3) / ome3 - a * rho2;
  } else {
    real cs2 = 1.0 / 3.0;
    real psi = 1. - EXPR(-rho);
    real psi2 = psi * psi;
    return cs2 * rho + cs2 * (real)o->p.G / 2 * psi2;
  }
}

/* dPsi, include/iteration_device.cuh:31-38 */
static real psi_of(const mlbmo* o, real rho) {
  if (o->p.carn_star) {
    real cs2 = 1.0 / 3.0;
    real pr = press(o, rho);
    return SQRTR(2.0 * (pr - cs2 * rho) / (cs2 * (real)o->p.G));
  }
  return 1. - EXPR(-rho);
}

static int bc_kind(const mlbmo* o, int x) {
  if (x < o->p.inlet_width) return 1;
  if (x >= o->lx - o->p.outlet_width) return 2;
  return 0;
}

mlbmo* SYM(create)(int lx, int ly, int lz, const mlbmo_params* p,
                   const float* rho_xyz, const uint8_t* fluid_xyz) {
  mlbmo* o = (mlbmo*)calloc(1, sizeof(mlbmo));
  if (!o) return NULL;
  o->lx = lx; o->ly = ly; o->lz = lz;
  o->n = (size_t)lx * ly * lz;
  o->p = *p;
  const real t0 = 1.0 / 3.0, t1 = 1.0 / 18.0, t2 = 1.0 / 36.0;
  const real tt[Q] = {t0, t1, t1, t1, t2, t2, t2, t2, t2, t2,
                      t1, t1, t1, t2, t2, t2, t2, t2, t2};
  memcpy(o->t, tt, sizeof tt);
  o->rho = (real*)calloc(o->n, sizeof(real));
  o->psi = (real*)calloc(o->n, sizeof(real));
  o->pressure = (real*)calloc(o->n, sizeof(real));
  o->force = (real*)calloc(3 * o->n, sizeof(real));
  o->vel = (real*)calloc(3 * o->n, sizeof(real));
  o->fa = (real*)calloc(Q * o->n, sizeof(real));
  o->fb = (real*)calloc(Q * o->n, sizeof(real));
  o->fluid = (uint8_t*)calloc(o->n, 1);
  if (!o->rho || !o->psi || !o->pressure || !o->force || !o->vel || !o->fa || !o->fb ||
      !o->fluid) {
    free(o);
    return NULL;
  }
  for (size_t k = 0; k < o->n; ++k) {
    o->rho[k] = (real)rho_xyz[k];
    o->fluid[k] = fluid_xyz[k] ? 1 : 0;
  }
  /* multiphaselbm_init, include/iteration_kernel.cuh:9-29 */
#pragma omp parallel for schedule(static)
  for (int x = 0; x < lx; ++x)
    for (int y = 0; y < ly; ++y)
      for (int z = 0; z < lz; ++z) {
        size_t k = idx(o, x, y, z);
        for (int i = 0; i < Q; ++i) {
          o->fa[k * Q + i] = o->t[i] * o->rho[k];
          o->fb[k * Q + i] = o->t[i] * o->rho[k];
        }
        if (o->fluid[k]) {
          o->psi[k] = psi_of(o, o->rho[k]);
          o->pressure[k] = press(o, o->rho[k]);
        } else {
          o->rho[k] = (real)o->p.rhos;
          o->psi[k] = psi_of(o, (real)o->p.rhos);
          o->force[3 * k] = o->force[3 * k + 1] = o->force[3 * k + 2] = 0;
        }
      }
  return o;
}

void SYM(destroy)(mlbmo* o) {
  if (!o) return;
  free(o->rho); free(o->psi); free(o->pressure); free(o->force); free(o->vel);
  free(o->fa); free(o->fb); free(o->fluid);
  free(o);
}

static void one_step(mlbmo* o, long step, int reverse, unsigned inject_type) {
  const int lx = o->lx, ly = o->ly, lz = o->lz;
  real* cf = o->fa; /* post-collision populations of the previous step */
  real* sf = o->fb; /* populations being built for this step */
  const real tau = (real)o->p.tau, G = (real)o->p.G;

  /* streaming + halfway bounce-back:
   * include/iteration_device.cuh:252-271, include/iteration_kernel.cuh:65-118 */
#pragma omp parallel for schedule(static)
  for (int x = 0; x < lx; ++x)
    for (int y = 0; y < ly; ++y)
      for (int z = 0; z < lz; ++z) {
        size_t k = idx(o, x, y, z);
        if (!o->fluid[k]) continue;
        sf[k * Q] = cf[k * Q];
        for (int i = 1; i < Q; ++i) {
          size_t s = idx(o, wrap(x - EX[i], lx), wrap(y - EY[i], ly),
                         wrap(z - EZ[i], lz));
          int opp = i > HALF ? i - HALF : i + HALF;
          sf[k * Q + i] = o->fluid[s] ? cf[s * Q + i] : cf[k * Q + opp];
        }
      }

  /* compute_density, include/iteration_device.cuh:40-63 */
#pragma omp parallel for schedule(static)
  for (int x = 0; x < lx; ++x)
    for (int y = 0; y < ly; ++y)
      for (int z = 0; z < lz; ++z) {
        size_t k = idx(o, x, y, z);
        if (!o->fluid[k]) continue;
        real d = 0.0;
        for (int i = 0; i < Q; ++i) d += sf[k * Q + i];
        /* a zero period (a division by zero in the reference) never injects */
        if (y < (real)o->p.inject_position * ly &&
            o->p.rho_inject_period != 0 &&
            (size_t)step % (size_t)o->p.rho_inject_period == 0) {
          real inc = (real)o->p.rho_increment;
          switch (inject_type) {
            case 0: d += inc * reverse; break;
            case 1: if (d < (real)o->p.rhol_spinodal) d += inc * reverse; break;
            case 2: if (d > (real)o->p.rhol_spinodal) d += inc * reverse; break;
          }
        }
        int bk = bc_kind(o, x);
        if (bk) d = (real)(bk == 1 ? o->p.rho_inlet : o->p.rho_outlet);
        o->rho[k] = d;
        o->pressure[k] = press(o, d);
        o->psi[k] = psi_of(o, o->rho[k]);
      }

  /* compute_force, compute_velocity, post_collision:
   * include/iteration_device.cuh:69-206 */
#pragma omp parallel for schedule(static)
  for (int x = 0; x < lx; ++x)
    for (int y = 0; y < ly; ++y)
      for (int z = 0; z < lz; ++z) {
        size_t k = idx(o, x, y, z);
        if (!o->fluid[k]) continue;
        real* f = sf + k * Q;
        if (bc_kind(o, x)) {
          for (int i = 0; i < Q; ++i) f[i] = o->t[i] * o->rho[k];
          o->force[3 * k] = o->force[3 * k + 1] = o->force[3 * k + 2] = 0;
          o->vel[3 * k] = o->vel[3 * k + 1] = o->vel[3 * k + 2] = 0;
          continue;
        }
        /* psi at x + e_i, in the reference's term order i = 1..18 */
        real pn[Q];
        for (int i = 1; i < Q; ++i)
          pn[i] = o->psi[idx(o, wrap(x + EX[i], lx), wrap(y + EY[i], ly),
                             wrap(z + EZ[i], lz))];
        real sx = o->t[1] * pn[1] * EX[1], sy = o->t[1] * pn[1] * EY[1],
             sz = o->t[1] * pn[1] * EZ[1];
        for (int i = 2; i < Q; ++i) {
          sx = sx + o->t[i] * pn[i] * EX[i];
          sy = sy + o->t[i] * pn[i] * EY[i];
          sz = sz + o->t[i] * pn[i] * EZ[i];
        }
        real Fx = -G * o->psi[k] * sx;
        real Fy = -G * o->psi[k] * sy;
        real Fz = -G * o->psi[k] * sz;
        o->force[3 * k] = Fx;
        o->force[3 * k + 1] = Fy;
        o->force[3 * k + 2] = Fz;

        real ux = 0.0, uy = 0.0, uz = 0.0;
        for (int i = 0; i < Q; ++i) {
          ux += f[i] * EX[i];
          uy += f[i] * EY[i];
          uz += f[i] * EZ[i];
        }
        ux += tau * Fx;
        uy += tau * Fy;
        uz += tau * Fz;
        real inv_rho = 1.0 / o->rho[k];
        ux *= inv_rho;
        uy *= inv_rho;
        uz *= inv_rho;
        o->vel[3 * k] = ux;
        o->vel[3 * k + 1] = uy;
        o->vel[3 * k + 2] = uz;
        real usq = ux * ux + uy * uy + uz * uz;
        real inv_tau = 1.0 / tau;
        for (int i = 0; i < Q; ++i) {
          real eu = EX[i] * ux + EY[i] * uy + EZ[i] * uz;
          f[i] += (o->t[i] * o->rho[k] *
                       (1.0 + 3.0 * eu + 4.5 * eu * eu - 1.5 * usq) -
                   f[i]) *
                  inv_tau;
        }
      }
  /* do_swap, include/iteration_kernel.cuh:44-48 */
  o->fa = sf;
  o->fb = cf;
}

void SYM(step)(mlbmo* o, int64_t step0, int32_t nsteps, int32_t reverse,
               uint32_t inject_type) {
  for (int32_t s = 0; s < nsteps; ++s)
    one_step(o, (long)(step0 + s), reverse, inject_type);
}

/* which: 0 rho, 1 pressure, 2 psi, 3 force [.][3], 4 post-collision
 * populations [.][19], 5 velocity u = (sum f e + tau F)/rho [.][3] of the
 * last step (include/iteration_device.cuh:181-203); copied out as `real`. */
int SYM(get)(const mlbmo* o, int32_t which, real* out) {
  switch (which) {
    case 0: memcpy(out, o->rho, o->n * sizeof(real)); return 0;
    case 1: memcpy(out, o->pressure, o->n * sizeof(real)); return 0;
    case 2: memcpy(out, o->psi, o->n * sizeof(real)); return 0;
    case 3: memcpy(out, o->force, 3 * o->n * sizeof(real)); return 0;
    case 4: memcpy(out, o->fa, Q * o->n * sizeof(real)); return 0;
    case 5: memcpy(out, o->vel, 3 * o->n * sizeof(real)); return 0;
  }
  return 1;
}

/* Phase statistics over fluid nodes as the reference computes them in
 * calc_cluster (src/multiphase_lbm.cu:240-275) and write_stats (:1061-1072):
 * out = {n_fluid, n_liquid, n_vapour, sum_p_liq, sum_p_vap, sum_rho_liq,
 *        sum_rho_vap, sum_rho_fluid (FP64), min_rho, max_rho, min_p, max_p} */
void SYM(phase_stats)(const mlbmo* o, double* out) {
  double nf = 0, nl = 0, nv = 0, pl = 0, pv = 0, rl = 0, rv = 0, mass = 0;
  double mn = 1e9, mx = -1e-9, pmn = 1e9, pmx = -1e-9;
  for (size_t k = 0; k < o->n; ++k) {
    if (!o->fluid[k]) continue;
    double r = o->rho[k], pr = o->pressure[k];
    nf += 1;
    mass += r;
    if (r > o->p.rhol_spinodal) { nl += 1; pl += pr; rl += r; }
    else if (r < o->p.rhog_spinodal) { nv += 1; pv += pr; rv += r; }
    if (r < mn) mn = r;
    if (r > mx) mx = r;
    if (pr < pmn) pmn = pr;
    if (pr > pmx) pmx = pr;
  }
  out[0] = nf; out[1] = nl; out[2] = nv; out[3] = pl; out[4] = pv;
  out[5] = rl; out[6] = rv; out[7] = mass; out[8] = mn; out[9] = mx;
  out[10] = pmn; out[11] = pmx;
}
