/*
 * track_oracle.c -- CPU oracle of probtrackx's simple mode on bedpostx samples.  TEST
 * INFRASTRUCTURE ONLY (loaded by tests/ as the checker of bpx_probtrack_dev; the product never
 * calls it).
 *
 * Restates, one particle at a time:
 *   Seedmanager::run            (streamlines.cc:1029-1120): both halves of a streamline from the
 *                               seed, kept halves, the streamline count (waytotal);
 *   Streamliner::streamline     (streamlines.cc:209-404): steps inside the mask, the path, the
 *                               waypoint, avoid (rubbish) and stop masks, the curvature stop,
 *                               the jump, the distance threshold;
 *   Counter::update_pathdist    (streamlines.cc:662-690): every voxel of a kept streamline counted
 *                               once (fdt_paths), per seed point with per_seed (ptx_simple.cc:50-62);
 *   Counter::update_seedcounts  (streamlines.cc:700-748): seeds to targets;
 *   Counter::update_matrix2_row (streamlines.cc:772-808): --omatrix2;
 *   Counter::update_matrix1     (streamlines.cc:751-770): --omatrix1, the per-seed path
 *                               distribution read at the seed-mask voxels;
 *   --prefdir                   (streamlines.cc:286-291, tractvolsx.h:209-225): the fibre closest
 *                               to a preferred direction per voxel after the first sample;
 *   Tractvolsx::sample          (tractvolsx.h:101-255): probabilistic rounding of the position,
 *                               a random posterior sample, the first fibre (fibst, randfib 1/2)
 *                               and afterwards the fibre closest to the current direction among
 *                               those with f > fibthresh, f for --usef;
 *   Particle::jump / testjump / check_dir / restart_reverse (particle.h), --modeuler's test
 *                               sample and mean direction, --loopcheck's coarse direction volume.
 * The reference draws from rand(); here every step's uniforms come from Philox-4x32-10 keyed by
 * the seed and counted by (particle, half, step), exactly as the GPU kernel draws them, and the
 * arithmetic is single precision in the reference's operation order, with the sine and cosine of
 * the GPU path (Cody-Waite reduction and the fitted quarter-period polynomials kSinQ/kCosQ of
 * bpx_device.cuh), so the oracle and the kernel follow identical paths.  MISCMATHS::round is taken
 * as floor(x + 0.5); sample positions are clamped to the grid (the reference reads its volume
 * there through newimage's boundary handling).  Compiled with -ffp-contract=off.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "bpx_oracle.h"

/* the quarter-period polynomial coefficients of bpx_device.cuh (generated by fdt_b200/polyfit.py);
 * tests/test_track_oracle.py checks that these literals equal the header's */
static const float kSinQ[3] = {-0.16666655f, 0.008332156f, -0.00019514632f};
static const float kCosQ[3] = {0.041666646f, -0.0013887362f, 2.443773e-05f};

static void sincos_quarter(float r, float* s, float* c) {
  const float u = r * r;
  float p = fmaf(u, kSinQ[2], kSinQ[1]);
  p = fmaf(u, p, kSinQ[0]);
  *s = fmaf(r * u, p, r);
  float q = fmaf(u, kCosQ[2], kCosQ[1]);
  q = fmaf(u, q, kCosQ[0]);
  q = fmaf(u, q, -0.5f);
  *c = fmaf(u, q, 1.0f);
}

static float flip_sign(float a, int flip) {
  uint32_t b;
  memcpy(&b, &a, 4);
  b ^= flip ? 0x80000000u : 0u;
  memcpy(&a, &b, 4);
  return a;
}

void orc_sincos_fast(float x, float* sn, float* cs) {
  const float k = rintf(x * 0.636619772f);
  float r = fmaf(-k, 1.57079637f, x);
  r = fmaf(-k, -4.37113883e-08f, r);
  r = fmaf(-k, -1.71512451e-15f, r);
  float s, c;
  sincos_quarter(r, &s, &c);
  const int q = (int)k;
  const int sw = (q & 1) != 0;
  const float a = sw ? c : s, b = sw ? s : c;
  *sn = flip_sign(a, (q & 2) != 0);
  *cs = flip_sign(b, ((q + 1) & 2) != 0);
}

static float u24(uint32_t x) { return (float)(x >> 8) * (1.0f / 16777216.0f); }

/* 8 uniforms in [0,1) for step `step` of half `half` of particle `pid` */
void orc_track_uniforms(uint64_t seed, uint64_t pid, int half, uint32_t step, float u[8]) {
  const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  for (int c = 0; c < 2; ++c) {
    const uint32_t ctr[4] = {(uint32_t)pid, (uint32_t)(pid >> 32), step, 0x80000000u | (uint32_t)(2 * half + c)};
    uint32_t r[4];
    orc_philox4x32_10(ctr, key, r);
    for (int i = 0; i < 4; ++i) u[4 * c + i] = u24(r[i]);
  }
}

static int rnd(float v) { return (int)floorf(v + 0.5f); }

typedef struct {
  const bpx_track_options* o;
  const bpx_track_volume* v;
  size_t nvox;
  float sx, sy, sz; /* steplength / voxel size */
} trk_t;

typedef struct {
  float x, y, z, rx, ry, rz, rxi, ryi, rzi;
  int jumped;
} part_t;

static int inside(const trk_t* T, int ix, int iy, int iz) {
  const bpx_track_volume* v = T->v;
  if (ix < 0 || iy < 0 || iz < 0 || ix >= v->nx || iy >= v->ny || iz >= v->nz) return 0;
  return v->mask[((size_t)iz * v->ny + iy) * v->nx + ix] > 0.f;
}

static int clampi(int a, int lo, int hi) { return a < lo ? lo : (a > hi ? hi : a); }

static size_t at(const trk_t* T, int k, int s, size_t vox) {
  return ((size_t)k * T->v->nsamples + s) * T->nvox + vox;
}

/* Tractvolsx::sample at position (x, y, z) with the particle's direction P->r and the preferred
 * direction pref of the step's voxel (zero without --prefdir): theta, phi and f */
static void sample(const trk_t* T, const part_t* P, float x, float y, float z, const float u[8], const float pref[3],
                   int* init_sample, int* fibst, float* th, float* ph, float* f) {
  const bpx_track_volume* v = T->v;
  const int cx = (int)ceilf(x), fx = (int)floorf(x);
  const int cy = (int)ceilf(y), fy = (int)floorf(y);
  const int cz = (int)ceilf(z), fz = (int)floorf(z);
  const float pcx = (cx == fx) ? 1.0f : (x - (float)fx) / (float)(cx - fx);
  const float pcy = (cy == fy) ? 1.0f : (y - (float)fy) / (float)(cy - fy);
  const float pcz = (cz == fz) ? 1.0f : (z - (float)fz) / (float)(cz - fz);
  const int nx_ = clampi(u[0] > pcx ? fx : cx, 0, v->nx - 1);
  const int ny_ = clampi(u[1] > pcy ? fy : cy, 0, v->ny - 1);
  const int nz_ = clampi(u[2] > pcz ? fz : cz, 0, v->nz - 1);
  const size_t vox = ((size_t)nz_ * v->ny + ny_) * v->nx + nx_;
  const int samp = clampi(rnd(u[3] * (float)(v->nsamples - 1)), 0, v->nsamples - 1);
  const int K = v->nfib;
  const float thr = T->o->fibthresh;
  float theta = 0.f, phi = 0.f;
  int fibind = 0;
  if (K > 1) {
    if (*init_sample) {
      if (T->o->randfib == 1) {
        int list[BPX_MAX_FIBRES], n = 0;
        for (int k = 0; k < K; ++k)
          if (v->f[at(T, k, samp, vox)] > thr) list[n++] = k;
        *fibst = n == 0 ? 0 : list[clampi(rnd(u[4] * (float)(n - 1)), 0, n - 1)];
      } else if (T->o->randfib == 2) {
        float fsum = 0.f;
        for (int k = 0; k < K; ++k) {
          const float ft = v->f[at(T, k, samp, vox)];
          if (ft > thr) fsum += ft;
        }
        if (fsum == 0.f) {
          *fibst = 0;
        } else {
          const float r = fsum * u[4];
          float cum = 0.f;
          for (int k = 0; k < K; ++k) {
            const float ft = v->f[at(T, k, samp, vox)];
            if (ft > thr) cum += ft;
            if (r <= cum) {
              *fibst = k;
              break;
            }
          }
        }
      }
      theta = v->th[at(T, *fibst, samp, vox)];
      phi = v->ph[at(T, *fibst, samp, vox)];
      *init_sample = 0;
    } else {
      /* the preferred direction, or where it is zero (always, without --prefdir) the current one */
      const int nopref = (fabsf(pref[0]) + fabsf(pref[1]) + fabsf(pref[2])) == 0.f;
      const float px = nopref ? P->rx : pref[0], py = nopref ? P->ry : pref[1], pz = nopref ? P->rz : pref[2];
      float dotmax = 0.f;
      for (int k = 0; k < K; ++k) {
        if (v->f[at(T, k, samp, vox)] > thr) {
          const float pht = v->ph[at(T, k, samp, vox)], tht = v->th[at(T, k, samp, vox)];
          float st, ct, sp, cp;
          orc_sincos_fast(tht, &st, &ct);
          orc_sincos_fast(pht, &sp, &cp);
          const float dot = fabsf(st * cp * px + st * sp * py + ct * pz);
          if (dot > dotmax) {
            dotmax = dot;
            theta = tht;
            phi = pht;
            fibind = k;
          }
        }
      }
      if (dotmax == 0.f) {
        theta = v->th[at(T, 0, samp, vox)];
        phi = v->ph[at(T, 0, samp, vox)];
      }
    }
  } else {
    theta = v->th[at(T, 0, samp, vox)];
    phi = v->ph[at(T, 0, samp, vox)];
  }
  *th = theta;
  *ph = phi;
  *f = T->o->usef ? v->f[at(T, fibind, samp, vox)] : 1.0f;
}

/* the 8 uniforms of a step's modified-Euler test sample (--modeuler): 0-3 its rounding and sample,
 * 4 the test jump's sign before the first jump */
void orc_track_uniforms_euler(uint64_t seed, uint64_t pid, int half, uint32_t step, float u[8]) {
  const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  for (int c = 0; c < 2; ++c) {
    const uint32_t ctr[4] = {(uint32_t)pid, (uint32_t)(pid >> 32), step, 0xC0000000u | (uint32_t)(2 * half + c)};
    uint32_t r[4];
    orc_philox4x32_10(ctr, key, r);
    for (int i = 0; i < 4; ++i) u[4 * c + i] = u24(r[i]);
  }
}

/* Particle::jump along the unit vector (rxn, ryn, rzn); the sign keeps the direction of travel, or is
 * drawn (u6) on the first jump */
static void jump_dir(const trk_t* T, part_t* P, float rxn, float ryn, float rzn, float u6) {
  const bpx_track_options* o = T->o;
  int sign, init = 0;
  if (P->jumped) {
    sign = (rxn * P->rx + ryn * P->ry + rzn * P->rz) > 0.f ? 1 : -1;
  } else {
    sign = u6 > 0.5f ? 1 : -1;
    P->jumped = 1;
    init = 1;
  }
  const float s = (float)sign;
  P->x += s * o->steplength / T->v->dx * rxn;
  P->y += s * o->steplength / T->v->dy * ryn;
  P->z += s * o->steplength / T->v->dz * rzn;
  P->rx = s * rxn;
  P->ry = s * ryn;
  P->rz = s * rzn;
  if (init) {
    P->rxi = P->rx;
    P->ryi = P->ry;
    P->rzi = P->rz;
  }
}

/* --loopcheck's volume of last directions on a 5x coarser grid (Streamliner::m_loopcheck,
 * streamlines.cc:112-116,248-263), cleared after every half */
typedef struct {
  int nx, ny, nz;
  float* dir; /* [nz][ny][nx][3] */
} loopvol_t;

/* one half of a streamline (Streamliner::streamline); appends the path's voxels to path[];
 * *flags accumulates the waypoint masks passed (over both halves of a particle); returns the
 * reject flag: 1 (entered the avoid mask, passed no waypoint, or shorter than distthresh), 2 (passed
 * some waypoints but not all), 0 */
/* --omatrix2: the tract-space voxel of a path position (vox_to_vox with the identity, then
 * MISCMATHS::round), or -1 off the tract-space grid */
static int64_t lr_voxel(const bpx_track_volume* v, float x, float y, float z) {
  /* vox_to_vox works in double (NEWMAT) and the result is rounded to float before MISCMATHS::round */
  const int lx = rnd((float)(((double)x * v->dx) / v->lr_dx)), ly = rnd((float)(((double)y * v->dy) / v->lr_dy)),
            lz = rnd((float)(((double)z * v->dz) / v->lr_dz));
  if (lx < 0 || ly < 0 || lz < 0 || lx >= v->lr_nx || ly >= v->lr_ny || lz >= v->lr_nz) return -1;
  return ((int64_t)lz * v->lr_ny + ly) * v->lr_nx + lx;
}

static int half_line(const trk_t* T, part_t* P, uint64_t pid, int h, int fibst0, float x0, float y0, float z0,
                     int64_t* path, int64_t* lrpath, int* npath, uint32_t* flags, loopvol_t* lc) {
  const bpx_track_options* o = T->o;
  const bpx_track_volume* v = T->v;
  int init_sample = 1, fibst = fibst0, avoided = 0;
  P->x = x0;
  P->y = y0;
  P->z = z0;
  float pathlength = 0.f;
  for (int it = 1; it <= o->nsteps / 2; ++it) {
    const int ix = rnd(P->x), iy = rnd(P->y), iz = rnd(P->z);
    if (!inside(T, ix, iy, iz)) break;  /* the reference's remaining steps change nothing */
    if (o->loopcheck) {
      /* stop where the path runs against the direction it last had in this coarse cell */
      const int lx = rnd(P->x / 5.0f), ly = rnd(P->y / 5.0f), lz = rnd(P->z / 5.0f);
      float* d = lc->dir + 3 * (((size_t)lz * lc->ny + ly) * lc->nx + lx);
      if (P->rx * d[0] + P->ry * d[1] + P->rz * d[2] < 0.f) break;
      d[0] = P->rx;
      d[1] = P->ry;
      d[2] = P->rz;
    }
    const int64_t vox = ((int64_t)iz * v->ny + iy) * v->nx + ix;
    if (v->waypoints) *flags |= v->waypoints[vox];
    if (v->m2_ncols > 0) lrpath[*npath] = lr_voxel(v, P->x, P->y, P->z);
    path[(*npath)++] = vox;
    pathlength += o->steplength;
    if (v->avoid && v->avoid[vox] != 0.f) {
      avoided = 1;
      break;
    }
    if (v->stop && v->stop[vox] != 0.f) break;
    float u[8], th, ph, f;
    float pref[3] = {0.f, 0.f, 0.f}; /* --prefdir at the rounded position (streamlines.cc:286-291) */
    if (v->prefdir)
      for (int c = 0; c < 3; ++c) pref[c] = v->prefdir[(size_t)c * T->nvox + (size_t)vox];
    orc_track_uniforms(o->seed, pid, h, (uint32_t)it, u);
    sample(T, P, P->x, P->y, P->z, u, pref, &init_sample, &fibst, &th, &ph, &f);
    if (f > u[5]) {
      float st, ct, sp, cp;
      orc_sincos_fast(th, &st, &ct);
      orc_sincos_fast(ph, &sp, &cp);
      const float rxn = cp * st, ryn = sp * st, rzn = ct;
      if (P->jumped && !(fabsf(rxn * P->rx + ryn * P->ry + rzn * P->rz) > o->c_thr)) break;
      if (th != 0.f && ph != 0.f) {
        if (!o->modeuler) {
          jump_dir(T, P, rxn, ryn, rzn, u[6]);
        } else {
          /* Particle::testjump, a sample there, and the jump along the mean of both directions
           * (mean_sph_pol, streamlines.cc:12-27, as the normalised sum or difference) */
          float w[8];
          orc_track_uniforms_euler(o->seed, pid, h, (uint32_t)it, w);
          int tsign;
          if (P->jumped)
            tsign = (rxn * P->rx + ryn * P->ry + rzn * P->rz) > 0.f ? 1 : -1;
          else
            tsign = w[4] > 0.5f ? 1 : -1;
          const float ts = (float)tsign;
          const float tx = P->x + ts * o->steplength / v->dx * rxn;
          const float ty = P->y + ts * o->steplength / v->dy * ryn;
          const float tz = P->z + ts * o->steplength / v->dz * rzn;
          float th2, ph2, f2;
          sample(T, P, tx, ty, tz, w, pref, &init_sample, &fibst, &th2, &ph2, &f2);
          float st2, ct2, sp2, cp2;
          orc_sincos_fast(th2, &st2, &ct2);
          orc_sincos_fast(ph2, &sp2, &cp2);
          const float bx = cp2 * st2, by = sp2 * st2, bz = ct2;
          const float same = (rxn * bx + ryn * by + rzn * bz) > 0.f ? 1.0f : -1.0f;
          const float mx = (rxn + same * bx) * 0.5f, my = (ryn + same * by) * 0.5f, mz = (rzn + same * bz) * 0.5f;
          const float n = sqrtf(mx * mx + my * my + mz * mz);
          if (n > 0.f)
            jump_dir(T, P, mx / n, my / n, mz / n, u[6]);
          else
            jump_dir(T, P, rxn, ryn, rzn, u[6]);
        }
      }
    }
  }
  if (o->loopcheck) memset(lc->dir, 0, sizeof(float) * 3 * (size_t)lc->nx * lc->ny * lc->nz);
  int rej = 0;
  if (v->nwaypoints > 0) {
    const uint32_t all = v->nwaypoints >= 32 ? 0xffffffffu : ((1u << v->nwaypoints) - 1u);
    const int passed = __builtin_popcount(*flags & all);
    rej = passed == 0 ? 1 : (passed < v->nwaypoints ? 2 : 0);
  }
  if (avoided) rej = 1;
  if (pathlength < o->distthresh) rej = 1;
  return rej;
}

/* Particles are independent: OpenMP threads take them in chunks, each with its own path, visit
 * stamps and loopcheck volume; the int32 counts and waytotal are integer sums, so the result does
 * not depend on the number of threads or the order. */
int orc_probtrack(const bpx_track_options* o, const bpx_track_volume* v, int nseeds, const float* seeds,
                  int32_t* paths, int64_t* waytotal) {
  trk_t T;
  T.o = o;
  T.v = v;
  T.nvox = (size_t)v->nx * v->ny * v->nz;
  const int half_steps = o->nsteps / 2;
  const int64_t total = (int64_t)nseeds * (int64_t)o->nparticles;
  uint32_t* counts = (uint32_t*)paths;
  int64_t kept = 0;
  int failed = 0;
#pragma omp parallel reduction(+ : kept) reduction(| : failed)
  {
    int64_t* path = (int64_t*)malloc(sizeof(int64_t) * (size_t)(2 * half_steps + 2));
    int64_t* lrpath = (int64_t*)malloc(sizeof(int64_t) * (size_t)(2 * half_steps + 2));
    const size_t lr_nvox = v->m2_ncols > 0 ? (size_t)v->lr_nx * v->lr_ny * v->lr_nz : 1;
    int64_t* stamp2 = (int64_t*)malloc(sizeof(int64_t) * lr_nvox); /* beenhere2 */
    int64_t* stamp = (int64_t*)malloc(sizeof(int64_t) * T.nvox);
    /* the coarse grid covers round(x / 5) for x in [-0.5, n - 0.5) */
    loopvol_t lc = {v->nx / 5 + 2, v->ny / 5 + 2, v->nz / 5 + 2, NULL};
    if (o->loopcheck) lc.dir = (float*)calloc(3 * (size_t)lc.nx * lc.ny * lc.nz, sizeof(float));
    const int ok = path && lrpath && stamp && stamp2 && (!o->loopcheck || lc.dir);
    if (!ok) failed = 1;
    if (ok) {
      for (size_t i = 0; i < T.nvox; ++i) stamp[i] = -1;
      for (size_t i = 0; i < lr_nvox; ++i) stamp2[i] = -1;
    }
#pragma omp for schedule(dynamic, 16)
    for (int64_t q = 0; q < total; ++q) {
      if (!ok) continue;
      const int s = (int)(q / o->nparticles);
      const uint64_t pid = (uint64_t)q;
      float u[8];
      orc_track_uniforms(o->seed, pid, 0, 0u, u); /* the particle's own draws: step 0 */
      int fibst = o->fibst - 1;
      if (o->randfib > 2) fibst = rnd(u[0] * (float)(v->nfib - 1));
      fibst = clampi(fibst, 0, v->nfib - 1);
      float x0 = seeds[3 * s], y0 = seeds[3 * s + 1], z0 = seeds[3 * s + 2];
      if (o->sampvox) {
        x0 += u[1] - 0.5f;
        y0 += u[2] - 0.5f;
        z0 += u[3] - 0.5f;
      }
      part_t P;
      memset(&P, 0, sizeof(P));
      int n1 = 0, n2 = 0;
      uint32_t flags = 0; /* waypoints passed, over both halves (Streamliner::reset clears them per particle) */
      const int rej1 = half_line(&T, &P, pid, 0, fibst, x0, y0, z0, path, lrpath, &n1, &flags, &lc);
      if (P.jumped) { /* Particle::restart_reverse */
        P.rx = -P.rxi;
        P.ry = -P.ryi;
        P.rz = -P.rzi;
      }
      const int rej2 = half_line(&T, &P, pid, 1, fibst, x0, y0, z0, path + n1, lrpath + n1, &n2, &flags, &lc);
      /* Seedmanager::run: the first half is kept on flag 0, or on 2 when the second half completes
       * the waypoints; the second half on flag 0 */
      const int fwd = (rej1 == 0 || rej1 == 2) && !(rej2 > 0 && rej1 > 0);
      const int bwd = rej2 == 0;
      if (!fwd && !bwd) continue;
      ++kept;
      /* Counter::update_pathdist over the kept halves in order: each distinct voxel adds 1, or
       * with --pd the d-th distinct voxel adds d (int32 sums wrap as the reference's int volume) */
      const int from = fwd ? 0 : n1, to = bwd ? n1 + n2 : n1;
      uint32_t d = 0, d2 = 0, tflags = 0;
      float clen = 0.f; /* path length along the counted path (Counter::update_seedcounts) */
      for (int i = from; i < to; ++i) {
        const int64_t vx = path[i];
        if (v->m2_ncols > 0 && lrpath[i] >= 0) {
          /* matrix2: each tract-space voxel once per streamline; column 0 and voxels outside the
           * mask are not counted (the reference's m_lookup2 test is "!= 0") */
          const int32_t col = v->m2_lookup[lrpath[i]];
          if (col > 0 && col < v->m2_ncols && stamp2[lrpath[i]] != (int64_t)pid) {
            stamp2[lrpath[i]] = (int64_t)pid;
            ++d2;
            const uint32_t add = o->pathdist ? d2 : 1u;
            uint32_t* m2 = (uint32_t*)v->matrix2;
#pragma omp atomic
            m2[(size_t)s * v->m2_ncols + col] += add;
          }
        }
        if (v->ntargets > 0) {
          /* seeds to targets: each target once per streamline, at its first entry, if the path is by
           * then at least distthresh long */
          const uint32_t tb = v->targets[vx] & ~tflags;
          if (tb) {
            if (clen >= o->distthresh)
              for (int m = 0; m < v->ntargets; ++m)
                if ((tb >> m) & 1u) {
#pragma omp atomic
                  v->seeds_to_targets[(size_t)m * nseeds + s] += 1;
                }
            tflags |= tb;
          }
        }
        clen += o->steplength;
        if (stamp[vx] != (int64_t)pid) {
          stamp[vx] = (int64_t)pid;
          ++d;
          const uint32_t add = o->pathdist ? d : 1u;
          const size_t at_vx = (o->per_seed ? (size_t)s * T.nvox : 0) + (size_t)vx;
#pragma omp atomic
          counts[at_vx] += add;
          if (v->m1_ncols > 0) {
            /* matrix1 (Counter::update_matrix1): the seed's path distribution read at the seed mask */
            const int32_t c1 = v->m1_lookup[vx];
            if (c1 >= 0 && c1 < v->m1_ncols) {
              uint32_t* m1 = (uint32_t*)v->matrix1;
#pragma omp atomic
              m1[(size_t)s * v->m1_ncols + c1] += add;
            }
          }
        }
      }
    }
    free(path);
    free(lrpath);
    free(stamp);
    free(stamp2);
    free(lc.dir);
  }
  if (failed) return 1;
  *waytotal += kept;
  return 0;
}
