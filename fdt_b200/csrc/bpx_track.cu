// bpx_track.cu -- probtrackx's simple mode on bedpostx samples (bpx_probtrack_dev).
//
// Replaces the per-particle loop of probtrackx (ptx_simple.cc:16-70 -> Seedmanager::run,
// streamlines.cc:1029-1120; Streamliner::streamline, streamlines.cc:209-404; Tractvolsx::sample,
// tractvolsx.h:101-255; Particle, particle.h) and its visit counting (Counter::update_pathdist,
// streamlines.cc:662-690).  One thread tracks one particle: both halves of its streamline from the
// seed, then adds 1 to fdt_paths in every voxel the kept halves passed through (once per voxel:
// a per-thread open-addressing table of the voxels already counted, entries stamped with the
// particle so no clearing is needed between particles) and 1 to waytotal.  With an avoid mask,
// waypoint masks or a distance threshold, the particle's halves are tracked once to learn which
// are kept, then the kept ones again (the same draws, so the same path) to count them.
//
// The work is a chain of dependent random gathers (the mask at the position and a posterior sample
// at a randomly rounded position, then the step), so the kernel is latency-bound: a persistent
// grid keeps as many particles in flight as the tables' workspace allows and every thread walks its
// particles in turn.  The samples are first repacked (pack_samples_kernel) so that one step reads
// one record of every fibre's direction and f instead of 3K scattered words, and forms no sine or
// cosine of the sampled angles.
//
// Arithmetic: single precision in the reference's operation order, no contraction into FMAs (this
// file is compiled with -fmad=false), sine and cosine from sincos_fast; random numbers from
// Philox-4x32-10 keyed by the seed, counted by (particle, half, step), eight uniforms per step.
// The CPU oracle (oracle/track_oracle.c) does the same operations and follows identical paths.
#include <cmath>
#include <cstdint>
#include <string>

#include "bpx.h"
#include "bpx_device.cuh"
#include "bpx_internal.h"

namespace bpx {
namespace {

constexpr int kTrackThreads = 64;
// 32 warps per SM to hide the gathers' latency: the launch bound holds a thread to 64 registers
// (no spills); measured on 1024 seeds x 5000 particles, 8 / 10 / 12 / 16 blocks per SM took
// 93.7 / 81.9 / 75.1 / 67.6 ms
constexpr int kTrackBlocksPerSm = 16;

// The options that carry state of their own compile into instantiations of the kernel of their
// own (a feature set), so each spills only what it must at the same launch bound: the plain form
// none (62 registers).  Measured on 1024 seeds x 5000 particles, 8 / 12 / 16 blocks per SM: 120 /
// 96 / 86 ms with --modeuler, 102 / 75 / 64 ms with --loopcheck, 86 / 64 / 57 ms with 3 targets,
// 255 / 219 / 204 ms with all of them and matrix2 (14 blocks: 204 ms).
constexpr int kFeatEuler = 1;  // --modeuler
constexpr int kFeatLoop = 2;   // --loopcheck
constexpr int kFeatCount = 4;  // seeds to targets, matrix2, matrix1
constexpr int kFeatPref = 8;   // --prefdir

struct TrackArgs {
  bpx_track_options o;
  bpx_track_volume v;
  size_t nvox;
  int nseeds;
  const float* seeds;
  int* paths;
  unsigned long long* waytotal;
  uint2* tables;       // [threads][1 << log2n] {voxel, stamp}
  int log2n;
  // [nvox][nsamples][pk4] float4: per fibre k, {v_x, v_y, v_z, f} with v = (sin th cos ph,
  // sin th sin ph, cos th) from sincos_fast; then one entry whose x holds bit k set when th_k and
  // ph_k are both non-zero (the reference takes no step along a sample with either exactly 0)
  const float4* packed;
  int pk4;  // float4 entries per (voxel, sample): nfib + 1
  // --loopcheck: per-thread tables [threads][1 << lc_log2n] of {coarse cell, stamp} and the
  // direction last seen there; the coarse grid is lcnx x lcny x lcnz (5x coarser)
  uint2* lc_keys;
  float4* lc_dirs;
  int lc_log2n;
  int lcnx, lcny;
  float sx, sy, sz;  // steplength / dx, dy, dz
  float lrx, lry, lrz;  // matrix2: dx / lr_dx, dy / lr_dy, dz / lr_dz
  uint64_t pid_begin;  // particles [pid_begin, pid_end) of this launch
  uint64_t pid_end;
};

__device__ __forceinline__ float u24(uint32_t x) { return (float)(x >> 8) * (1.0f / 16777216.0f); }

// block c (0 or 1) of a step's uniforms: u[4c .. 4c+3]
__device__ __forceinline__ void uniform_block(uint64_t seed, uint64_t pid, int half, uint32_t step, int c,
                                              float (&u)[8]) {
  const uint2 key = make_uint2((uint32_t)seed, (uint32_t)(seed >> 32));
  const uint4 r = philox4x32_10(make_uint4((uint32_t)pid, (uint32_t)(pid >> 32), step, 0x80000000u | (uint32_t)(2 * half + c)), key);
  u[4 * c + 0] = u24(r.x);
  u[4 * c + 1] = u24(r.y);
  u[4 * c + 2] = u24(r.z);
  u[4 * c + 3] = u24(r.w);
}

__device__ __forceinline__ void track_uniforms(uint64_t seed, uint64_t pid, int half, uint32_t step, float (&u)[8]) {
  uniform_block(seed, pid, half, step, 0, u);
  uniform_block(seed, pid, half, step, 1, u);
}

// the uniforms of a step's modified-Euler test sample: 0-3 its rounding and sample, 4 the test
// jump's sign before the first jump (the second block only when `second`; else 4-7 are zero)
__device__ __forceinline__ void euler_uniforms(uint64_t seed, uint64_t pid, int half, uint32_t step, bool second,
                                               float (&u)[8]) {
  const uint2 key = make_uint2((uint32_t)seed, (uint32_t)(seed >> 32));
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    if (c == 1 && !second) {
      u[4] = u[5] = u[6] = u[7] = 0.f;
      break;
    }
    const uint4 r = philox4x32_10(make_uint4((uint32_t)pid, (uint32_t)(pid >> 32), step, 0xC0000000u | (uint32_t)(2 * half + c)), key);
    u[4 * c + 0] = u24(r.x);
    u[4 * c + 1] = u24(r.y);
    u[4 * c + 2] = u24(r.z);
    u[4 * c + 3] = u24(r.w);
  }
}

__device__ __forceinline__ int rnd(float v) { return (int)floorf(v + 0.5f); }
__device__ __forceinline__ int clampi(int a, int lo, int hi) { return a < lo ? lo : (a > hi ? hi : a); }

struct Particle {
  float x, y, z, rx, ry, rz, rxi, ryi, rzi;
  bool jumped;
};

// Particle::restart_reverse: the second half starts from the seed against the first half's first step
__device__ __forceinline__ void reverse(Particle& P) {
  if (P.jumped) {
    P.rx = -P.rxi;
    P.ry = -P.ryi;
    P.rz = -P.rzi;
  }
}

// Particle::jump along the unit vector (rxn, ryn, rzn): the sign keeps the direction of travel, or
// is drawn (u6) on the first jump
__device__ __forceinline__ void jump_dir(Particle& P, const TrackArgs& a, float rxn, float ryn, float rzn, float u6) {
  int sign;
  bool init = false;
  if (P.jumped) {
    sign = (rxn * P.rx + ryn * P.ry + rzn * P.rz) > 0.f ? 1 : -1;
  } else {
    sign = u6 > 0.5f ? 1 : -1;
    P.jumped = true;
    init = true;
  }
  const float s = (float)sign;
  // (s * steplength) / dx equals s * (steplength / dx) exactly for s = +-1: the quotients are
  // formed once per launch (TrackArgs::sx, sy, sz)
  P.x += s * a.sx * rxn;
  P.y += s * a.sy * ryn;
  P.z += s * a.sz * rzn;
  P.rx = s * rxn;
  P.ry = s * ryn;
  P.rz = s * rzn;
  if (init) {
    P.rxi = P.rx;
    P.ryi = P.ry;
    P.rzi = P.rz;
  }
}

// what the counting passes of one particle carry over its kept halves: the path length so far on
// the counted path, the targets already entered, the particle's seed, the tract-space columns
// counted so far (--omatrix2 with --pd)
struct Counted {
  float length;
  uint32_t tflags;
  int seed;
  int nvisit2;
};

// --omatrix2's tract-space voxel keys share the visit table with the diffusion voxels
constexpr uint32_t kLrKey = 0x80000000u;

// Rounding of a quotient without the division: q, a float product within 3e-7 |q| of the exact
// quotient, decides floor(quotient + 1/2) wherever it lies farther than 1e-5 (|q| + 1) from a
// rounding boundary k + 1/2 (the quotient, and its correctly rounded float, then lie on the same
// side of it); returns false where it does not, and the caller forms the quotient itself.
__device__ __forceinline__ bool round_clear(float q, int& r) {
  r = (int)floorf(q + 0.5f);
  return fabsf((q - floorf(q)) - 0.5f) > 1e-5f * (fabsf(q) + 1.0f);
}

// --omatrix2's tract-space coordinate: round(float(x * d / lr_d)) as the reference forms it
// (vox_to_vox in double, the result rounded to float, then MISCMATHS::round); ratio = d / lr_d
__device__ __forceinline__ int lr_round(float x, float d, float lr_d, float ratio) {
  int r;
  if (round_clear(x * ratio, r)) return r;
  return rnd((float)(((double)x * (double)d) / (double)lr_d));
}

// --loopcheck's coarse coordinate round(x / 5)
__device__ __forceinline__ int lc_round(float x) {
  int r;
  if (round_clear(x * 0.2f, r)) return r;
  return rnd(x / 5.0f);
}

struct Tracker {
  const TrackArgs& a;
  uint2* tab;
  uint32_t stamp;
  int* paths;  // the volume this particle's visits go to (its seed's with per_seed)
  uint2* lck;        // this thread's loopcheck table
  float4* lcd;
  uint32_t lc_stamp;  // one per tracked half (the tables are cleared per launch)

  // --loopcheck: the direction stored for coarse cell `cell` this half (zero if none)
  __device__ float3 loop_get(uint32_t cell) const {
    const uint32_t mask = (1u << a.lc_log2n) - 1u;
    uint32_t h = (cell * 2654435761u) >> (32 - a.lc_log2n);
    for (uint32_t probe = 0; probe <= mask; ++probe) {
      const uint2 e = lck[h];
      if (e.y != lc_stamp) break;  // an empty entry ends the probe sequence: not stored
      if (e.x == cell) {
        const float4 o = lcd[h];
        return make_float3(o.x, o.y, o.z);
      }
      h = (h + 1u) & mask;
    }
    return make_float3(0.f, 0.f, 0.f);
  }
  // --loopcheck: stores d as the direction of coarse cell `cell` this half
  __device__ void loop_put(uint32_t cell, float3 d) const {
    const uint32_t mask = (1u << a.lc_log2n) - 1u;
    uint32_t h = (cell * 2654435761u) >> (32 - a.lc_log2n);
    for (uint32_t probe = 0; probe <= mask; ++probe) {
      const uint2 e = lck[h];
      if (e.y != lc_stamp || e.x == cell) {
        lck[h] = make_uint2(cell, lc_stamp);
        lcd[h] = make_float4(d.x, d.y, d.z, 0.f);
        return;
      }
      h = (h + 1u) & mask;
    }  // unreachable: the table holds twice the cells of a half
  }

  // the sample record of voxel `svox`, sample `samp`: every fibre's direction and f, and the
  // non-zero-angle bits
  struct Sample {
    float vx[BPX_MAX_FIBRES], vy[BPX_MAX_FIBRES], vz[BPX_MAX_FIBRES], f[BPX_MAX_FIBRES];
    uint32_t moves;  // bit k: th_k != 0 and ph_k != 0
  };
  __device__ void load_record(size_t svox, int samp, Sample& S) const {
    // one 32- to 64-byte record (one or two sectors)
    const float4* rec = a.packed + ((size_t)svox * a.v.nsamples + samp) * a.pk4;
    const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
    float4 r[BPX_MAX_FIBRES + 1];
#pragma unroll
    for (int q = 0; q <= BPX_MAX_FIBRES; ++q) r[q] = a.pk4 > q ? __ldg(rec + q) : zero;
    float4 fl = r[1];
#pragma unroll
    for (int k = 0; k < BPX_MAX_FIBRES; ++k) {
      S.vx[k] = r[k].x;
      S.vy[k] = r[k].y;
      S.vz[k] = r[k].z;
      S.f[k] = r[k].w;
      if (a.pk4 == k + 2) fl = r[k + 1];
    }
    S.moves = __float_as_uint(fl.x);
  }

  // first visit of `vox` by this particle: true (and the voxel is recorded)
  __device__ bool first_visit(uint32_t vox) const {
    const uint32_t mask = (1u << a.log2n) - 1u;
    uint32_t h = (vox * 2654435761u) >> (32 - a.log2n);
    for (uint32_t probe = 0; probe <= mask; ++probe) {
      const uint2 e = tab[h];
      if (e.y != stamp) {
        tab[h] = make_uint2(vox, stamp);
        return true;
      }
      if (e.x == vox) return false;
      h = (h + 1u) & mask;
    }
    return false;  // unreachable: the table holds twice the longest path
  }

  // The voxel and posterior sample a step reads (the probabilistic rounding of Tractvolsx::sample):
  // depends only on the position and the step's uniforms, so its loads can be issued together
  // with the mask's.
  __device__ void locate(float x, float y, float z, const float (&u)[8], size_t& vox, int& samp) const {
    const bpx_track_volume& v = a.v;
    const int cx = (int)ceilf(x), fx = (int)floorf(x);
    const int cy = (int)ceilf(y), fy = (int)floorf(y);
    const int cz = (int)ceilf(z), fz = (int)floorf(z);
    // (x - fx) / (cx - fx) with cx - fx = 1 whenever it is formed: the quotient is x - fx exactly
    const float pcx = (cx == fx) ? 1.0f : (x - (float)fx);
    const float pcy = (cy == fy) ? 1.0f : (y - (float)fy);
    const float pcz = (cz == fz) ? 1.0f : (z - (float)fz);
    const int nx_ = clampi(u[0] > pcx ? fx : cx, 0, v.nx - 1);
    const int ny_ = clampi(u[1] > pcy ? fy : cy, 0, v.ny - 1);
    const int nz_ = clampi(u[2] > pcz ? fz : cz, 0, v.nz - 1);
    vox = ((size_t)nz_ * v.ny + ny_) * v.nx + nx_;
    samp = clampi(rnd(u[3] * (float)(v.nsamples - 1)), 0, v.nsamples - 1);
  }

  // The fibre choice of Tractvolsx::sample on the voxel's sample: the chosen fibre's direction
  // (r), whether its angles are both non-zero (moves) and f (1 without --usef)
  __device__ void choose(const Particle& P, const float (&u)[8], const Sample& S, float3 pref, bool& init_sample,
                         int& fibst, float3& r, bool& moves, float& f) const {
    const int K = a.v.nfib;
    const float thr = a.o.fibthresh;
    int sel = 0, fibind = 0;
    if (K > 1) {
      if (init_sample) {
        if (a.o.randfib == 1) {
          int list[BPX_MAX_FIBRES], n = 0;
#pragma unroll
          for (int k = 0; k < BPX_MAX_FIBRES; ++k)
            if (k < K && S.f[k] > thr) list[n++] = k;
          fibst = n == 0 ? 0 : list[clampi(rnd(u[4] * (float)(n - 1)), 0, n - 1)];
        } else if (a.o.randfib == 2) {
          float fsum = 0.f;
#pragma unroll
          for (int k = 0; k < BPX_MAX_FIBRES; ++k)
            if (k < K && S.f[k] > thr) fsum += S.f[k];
          if (fsum == 0.f) {
            fibst = 0;
          } else {
            const float rr = fsum * u[4];
            float cum = 0.f;
            bool found = false;
#pragma unroll
            for (int k = 0; k < BPX_MAX_FIBRES; ++k) {
              if (k < K && !found) {
                if (S.f[k] > thr) cum += S.f[k];
                if (rr <= cum) {
                  fibst = k;
                  found = true;
                }
              }
            }
          }
        }
        sel = fibst;
        init_sample = false;
      } else {
        // the preferred direction of the step's voxel, or where it is zero (always, without
        // --prefdir) the current direction; |sin th cos ph px + sin th sin ph py + cos th pz| in the
        // reference's order
        const bool nopref = (fabsf(pref.x) + fabsf(pref.y) + fabsf(pref.z)) == 0.f;
        const float px = nopref ? P.rx : pref.x, py = nopref ? P.ry : pref.y, pz = nopref ? P.rz : pref.z;
        float dotmax = 0.f;
#pragma unroll
        for (int k = 0; k < BPX_MAX_FIBRES; ++k) {
          if (k < K && S.f[k] > thr) {
            const float dot = fabsf(S.vx[k] * px + S.vy[k] * py + S.vz[k] * pz);
            if (dot > dotmax) {
              dotmax = dot;
              sel = k;
              fibind = k;
            }
          }
        }
        if (dotmax == 0.f) sel = 0;
      }
    }
    r = make_float3(S.vx[0], S.vy[0], S.vz[0]);
    float ff = S.f[0];
#pragma unroll
    for (int k = 1; k < BPX_MAX_FIBRES; ++k) {
      if (k == sel) r = make_float3(S.vx[k], S.vy[k], S.vz[k]);
      if (k == fibind) ff = S.f[k];
    }
    moves = (S.moves >> sel) & 1u;
    f = a.o.usef ? ff : 1.0f;
  }

  // Streamliner::streamline for one half; counts the path's first visits when `count` (with --pd
  // the d-th distinct voxel of the particle adds d; nvisit carries d over the kept halves).  `flags`
  // accumulates the waypoint masks passed (over both halves of a particle).  Returns the reject
  // flag: 1 (entered the avoid mask, passed no waypoint, or shorter than distthresh), 2 (passed
  // some waypoints but not all), 0.
  // FEAT: the feature set compiled in (kFeatEuler, kFeatLoop, kFeatCount)
  template <int FEAT>
  __device__ int half_line(Particle& P, uint64_t pid, int h, int fibst0, float x0, float y0, float z0,
                           bool count, uint32_t& flags, int& nvisit, Counted& cnt) {
    const bpx_track_options& o = a.o;
    const bpx_track_volume& v = a.v;
    bool init_sample = true, avoided = false;
    int fibst = fibst0;
    P.x = x0;
    P.y = y0;
    P.z = z0;
    float pathlength = 0.f;
    const int K = v.nfib;
    // a step of steplength mm mostly stays in the voxel of the step before, which is counted
    // already: the visit table is probed only when the voxel changes
    uint32_t last = 0xffffffffu, last_lr = 0xffffffffu;
    ++lc_stamp;  // every tracked half starts with an empty loopcheck volume
    // --loopcheck: the coarse cell of the step before and the direction stored for it since; the
    // table is read and written only when the cell changes (about every 20 steps of 0.5 mm in 2 mm
    // voxels), which stores and finds the same directions as a table access every step
    uint32_t lc_cell = 0xffffffffu;
    float3 lc_dir = make_float3(0.f, 0.f, 0.f);
    for (int it = 1; it <= o.nsteps / 2; ++it) {
      const int ix = rnd(P.x), iy = rnd(P.y), iz = rnd(P.z);
      // this step's uniforms and sampled voxel, then the masks at the position and every fibre's
      // sample in one round of loads (the reference reads them only inside the mask: same values)
      // this step's uniforms: the first block always (rounding, sample); the second (randfib's
      // draw, the --usef test, the first jump's sign) only while one of its draws can be used
      float u[8], f;
      uniform_block(o.seed, pid, h, (uint32_t)it, 0, u);
      if (o.usef || !P.jumped || (init_sample && K > 1 && (o.randfib == 1 || o.randfib == 2))) {
        uniform_block(o.seed, pid, h, (uint32_t)it, 1, u);
      } else {
        u[4] = u[5] = u[6] = u[7] = 0.f;  // f is 1 without --usef, so the step is taken
      }
      size_t svox;
      int samp;
      locate(P.x, P.y, P.z, u, svox, samp);
      const bool in_grid = ix >= 0 && iy >= 0 && iz >= 0 && ix < v.nx && iy < v.ny && iz < v.nz;
      const uint32_t vox = in_grid ? (uint32_t)(((size_t)iz * v.ny + iy) * v.nx + ix) : 0u;
      const float m = __ldg(v.mask + vox);
      const uint32_t way = v.waypoints ? __ldg(v.waypoints + vox) : 0u;
      float3 pref = make_float3(0.f, 0.f, 0.f);  // --prefdir at the rounded position
      if ((FEAT & kFeatPref) && v.prefdir)
        pref = make_float3(__ldg(v.prefdir + vox), __ldg(v.prefdir + a.nvox + vox), __ldg(v.prefdir + 2 * a.nvox + vox));
      // what the counting below reads, in the same round: the target bits of a new voxel, the
      // matrix2 column of a new tract-space voxel (lr: its index, or ~0 off the tract-space grid)
      uint32_t tgt = 0u, lr = 0xffffffffu;
      int col = 0;
      if ((FEAT & kFeatCount) && count) {
        if (v.ntargets > 0 && vox != last) tgt = __ldg(v.targets + vox);
        if (v.m2_ncols > 0) {
          const int lx = lr_round(P.x, v.dx, v.lr_dx, a.lrx);
          const int ly = lr_round(P.y, v.dy, v.lr_dy, a.lry);
          const int lz = lr_round(P.z, v.dz, v.lr_dz, a.lrz);
          if (lx >= 0 && ly >= 0 && lz >= 0 && lx < v.lr_nx && ly < v.lr_ny && lz < v.lr_nz) {
            lr = ((uint32_t)lz * (uint32_t)v.lr_ny + (uint32_t)ly) * (uint32_t)v.lr_nx + (uint32_t)lx;
            if (lr != last_lr) col = __ldg(v.m2_lookup + lr);
          }
        }
      }
      const bool avoid = v.avoid && __ldg(v.avoid + vox) != 0.f;
      const bool stop = v.stop && __ldg(v.stop + vox) != 0.f;
      Sample S;
      load_record(svox, samp, S);
      if (!(in_grid && m > 0.f)) break;  // the reference's remaining steps change nothing
      if ((FEAT & kFeatLoop) && o.loopcheck) {
        // stop where the path runs against the direction it last had in this coarse cell
        const int lx = lc_round(P.x), ly = lc_round(P.y), lz = lc_round(P.z);
        const uint32_t cell = ((uint32_t)lz * (uint32_t)a.lcny + (uint32_t)ly) * (uint32_t)a.lcnx + (uint32_t)lx;
        float3 old = lc_dir;
        if (cell != lc_cell) {
          if (lc_cell != 0xffffffffu) loop_put(lc_cell, lc_dir);
          old = loop_get(cell);
          lc_cell = cell;
        }
        if (P.rx * old.x + P.ry * old.y + P.rz * old.z < 0.f) break;
        lc_dir = make_float3(P.rx, P.ry, P.rz);
      }
      flags |= way;
      if (count && vox != last) {
        last = vox;
        if (first_visit(vox)) {
          const int add = o.pathdist ? ++nvisit : 1;
          atomicAdd(paths + vox, add);
          if ((FEAT & kFeatCount) && v.m1_ncols > 0) {
            // --omatrix1: a seed-mask voxel's fdt_paths count also goes to the seed's row
            const int c1 = __ldg(v.m1_lookup + vox);
            if (c1 >= 0 && c1 < v.m1_ncols) atomicAdd(v.matrix1 + (size_t)cnt.seed * v.m1_ncols + c1, add);
          }
        }
        if ((FEAT & kFeatCount) && v.ntargets > 0) {
          // a target is counted at its first entry on the counted path (a voxel change), if the path
          // is by then at least distthresh long (Counter::update_seedcounts)
          const uint32_t tb = tgt & ~cnt.tflags;
          if (tb) {
            if (cnt.length >= o.distthresh)
              for (uint32_t b = tb; b; b &= b - 1) atomicAdd(v.seeds_to_targets + (size_t)(__ffs(b) - 1) * a.nseeds + cnt.seed, 1);
            cnt.tflags |= tb;
          }
        }
      }
      if ((FEAT & kFeatCount) && count && lr != 0xffffffffu && lr != last_lr) {
        // --omatrix2: the tract-space voxel of the position, counted once per particle when its
        // column is not 0 (Counter::update_matrix2_row); it can change inside a diffusion voxel
        last_lr = lr;
        if (col > 0 && col < v.m2_ncols && first_visit(lr | kLrKey))
          atomicAdd(v.matrix2 + (size_t)cnt.seed * v.m2_ncols + col, o.pathdist ? ++cnt.nvisit2 : 1);
      }
      if ((FEAT & kFeatCount) && count) cnt.length += o.steplength;
      pathlength += o.steplength;
      if (avoid) {
        avoided = true;
        break;
      }
      if (stop) break;
      float3 rn;
      bool moves;
      choose(P, u, S, pref, init_sample, fibst, rn, moves, f);
      if (f > u[5]) {
        // (cos ph sin th, sin ph sin th, cos th): the record's vector, products commuted
        const float rxn = rn.x, ryn = rn.y, rzn = rn.z;
        if (P.jumped && !(fabsf(rxn * P.rx + ryn * P.ry + rzn * P.rz) > o.c_thr)) break;
        if (moves) {
          if (!(FEAT & kFeatEuler) || !o.modeuler) {
            jump_dir(P, a, rxn, ryn, rzn, u[6]);
          } else {
            // Particle::testjump, a sample there, and the jump along the mean of both directions
            // (mean_sph_pol, streamlines.cc:12-27, as the normalised sum or difference)
            float w[8];
            euler_uniforms(o.seed, pid, h, (uint32_t)it, !P.jumped, w);
            int tsign;
            if (P.jumped)
              tsign = (rxn * P.rx + ryn * P.ry + rzn * P.rz) > 0.f ? 1 : -1;
            else
              tsign = w[4] > 0.5f ? 1 : -1;
            const float ts = (float)tsign;
            const float tx = P.x + ts * a.sx * rxn;
            const float ty = P.y + ts * a.sy * ryn;
            const float tz = P.z + ts * a.sz * rzn;
            size_t tvox;
            int tsamp;
            locate(tx, ty, tz, w, tvox, tsamp);
            Sample T2;
            load_record(tvox, tsamp, T2);
            float3 b;
            bool moves2;
            float f2;
            choose(P, w, T2, pref, init_sample, fibst, b, moves2, f2);
            const float bx = b.x, by = b.y, bz = b.z;
            const float same = (rxn * bx + ryn * by + rzn * bz) > 0.f ? 1.0f : -1.0f;
            const float mx = (rxn + same * bx) * 0.5f, my = (ryn + same * by) * 0.5f, mz = (rzn + same * bz) * 0.5f;
            const float n = sqrtf(mx * mx + my * my + mz * mz);
            if (n > 0.f)
              jump_dir(P, a, mx / n, my / n, mz / n, u[6]);
            else
              jump_dir(P, a, rxn, ryn, rzn, u[6]);
          }
        }
      }
    }
    int rej = 0;
    if (v.nwaypoints > 0) {
      const uint32_t all = v.nwaypoints >= 32 ? 0xffffffffu : ((1u << v.nwaypoints) - 1u);
      const int passed = __popc(flags & all);
      rej = passed == 0 ? 1 : (passed < v.nwaypoints ? 2 : 0);
    }
    if (avoided || pathlength < o.distthresh) rej = 1;
    return rej;
  }
};

template <int FEAT>
__global__ void __launch_bounds__(kTrackThreads, kTrackBlocksPerSm) track_kernel(TrackArgs a) {
  const uint64_t threads = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  Tracker T{a, a.tables + (t << a.log2n), 0u, a.paths, nullptr, nullptr, 0u};
  if (a.o.loopcheck) {
    T.lck = a.lc_keys + (t << a.lc_log2n);
    T.lcd = a.lc_dirs + (t << a.lc_log2n);
  }
  unsigned long long kept = 0;
  // a half's fate waits on its length (distthresh), on the avoid mask, or on the waypoints both
  // halves passed (Seedmanager::run keeps a first half with reject flag 2 when the second half
  // completes the waypoints)
  const bool decide = a.o.distthresh > 0.f || a.v.avoid != nullptr || a.v.nwaypoints > 0;
  for (uint64_t pid = a.pid_begin + t; pid < a.pid_end; pid += threads) {
    T.stamp = (uint32_t)(pid - a.pid_begin) + 1u;
    const int s = (int)(pid / (uint64_t)a.o.nparticles);
    if (a.o.per_seed) T.paths = a.paths + (size_t)s * a.nvox;
    float u0[8];
    track_uniforms(a.o.seed, pid, 0, 0u, u0);  // the particle's own draws: step 0
    int fibst = a.o.fibst - 1;
    if (a.o.randfib > 2) fibst = rnd(u0[0] * (float)(a.v.nfib - 1));
    fibst = clampi(fibst, 0, a.v.nfib - 1);
    float x0 = a.seeds[3 * s], y0 = a.seeds[3 * s + 1], z0 = a.seeds[3 * s + 2];
    if (a.o.sampvox) {
      x0 += u0[1] - 0.5f;
      y0 += u0[2] - 0.5f;
      z0 += u0[3] - 0.5f;
    }
    Particle P{};
    uint32_t flags = 0;  // waypoints passed by both halves (Streamliner::reset clears them per particle)
    int nvisit = 0;      // distinct voxels counted so far (the first half's before the second's)
    Counted cnt{0.f, 0u, s, 0};
    if (decide) {  // whether a half counts is known only once both halves have ended: track, then count
      const Particle P0 = P;
      const int rej1 = T.template half_line<FEAT>(P, pid, 0, fibst, x0, y0, z0, false, flags, nvisit, cnt);
      reverse(P);
      const Particle P1 = P;
      const int rej2 = T.template half_line<FEAT>(P, pid, 1, fibst, x0, y0, z0, false, flags, nvisit, cnt);
      const bool fwd = (rej1 == 0 || rej1 == 2) && !(rej2 > 0 && rej1 > 0), bwd = rej2 == 0;
      uint32_t unused = 0;
      if (fwd) {
        Particle Q = P0;
        T.template half_line<FEAT>(Q, pid, 0, fibst, x0, y0, z0, true, unused, nvisit, cnt);
      }
      if (bwd) {
        Particle Q = P1;
        T.template half_line<FEAT>(Q, pid, 1, fibst, x0, y0, z0, true, unused, nvisit, cnt);
      }
      if (fwd || bwd) ++kept;
    } else {  // every half is kept: count as it goes
      T.template half_line<FEAT>(P, pid, 0, fibst, x0, y0, z0, true, flags, nvisit, cnt);
      reverse(P);
      T.template half_line<FEAT>(P, pid, 1, fibst, x0, y0, z0, true, flags, nvisit, cnt);
      ++kept;
    }
  }
  // waytotal: one atomic per warp
  for (int o = 16; o >= 1; o >>= 1) kept += __shfl_xor_sync(0xffffffffu, kept, o);
  if ((threadIdx.x & 31) == 0 && kept) atomicAdd(a.waytotal, kept);
}

// The samples [K][nsamples][nvox] of th, ph and f repacked as one record per (voxel, sample)
// (TrackArgs::packed): a 32 x 32 tile of (voxel, sample) per block, read along voxels and written
// along samples through shared memory, so both sides are coalesced.  Each fibre's direction is
// formed here once, with the sine and cosine every step would otherwise form again.
constexpr int kPackTile = 32;
__global__ void __launch_bounds__(256) pack_samples_kernel(const float* __restrict__ th, const float* __restrict__ ph,
                                                           const float* __restrict__ f, int K, int ns, size_t nvox,
                                                           int pk4, float4* __restrict__ out) {
  __shared__ float tile[3 * BPX_MAX_FIBRES][kPackTile][kPackTile + 1];
  const size_t v0 = (size_t)blockIdx.x * kPackTile;
  const int s0 = blockIdx.y * kPackTile;
  const int tx = threadIdx.x, ty = threadIdx.y;
  for (int c = 0; c < 3 * K; ++c) {
    const float* src = (c % 3 == 0) ? th : (c % 3 == 1) ? ph : f;
    const int k = c / 3;
    for (int j = ty; j < kPackTile; j += blockDim.y) {
      const int smp = s0 + j;
      const size_t vx = v0 + tx;
      tile[c][j][tx] = (smp < ns && vx < nvox) ? src[((size_t)k * ns + smp) * nvox + vx] : 0.f;
    }
  }
  __syncthreads();
  for (int i = ty; i < kPackTile; i += blockDim.y) {
    const size_t vx = v0 + i;
    const int smp = s0 + tx;
    if (vx >= nvox || smp >= ns) continue;
    float4* dst = out + (vx * ns + smp) * pk4;
    uint32_t moves = 0;
    for (int k = 0; k < K; ++k) {
      const float t = tile[3 * k][tx][i], p = tile[3 * k + 1][tx][i];
      float st, ct, sp, cp;
      sincos_fast(t, st, ct);
      sincos_fast(p, sp, cp);
      dst[k] = make_float4(st * cp, st * sp, ct, tile[3 * k + 2][tx][i]);
      if (t != 0.f && p != 0.f) moves |= 1u << k;
    }
    dst[K] = make_float4(__uint_as_float(moves), 0.f, 0.f, 0.f);
  }
}

bpx_status check_track(const bpx_track_options* o, const bpx_track_volume* v, int32_t nseeds, const float* seeds,
                       const int32_t* paths, const int64_t* waytotal) {
  if (!o || !v) return api_fail(BPX_ERR_INVALID_ARG, "bpx_probtrack_dev: opts or vol is NULL");
  if (o->nparticles < 1 || o->nsteps < 2 || o->nsteps > (1 << 20))
    return api_fail(BPX_ERR_INVALID_ARG, "bpx_probtrack_dev: nparticles must be >= 1 and nsteps in 2..2^20");
  if (!(o->steplength > 0.f) || !(o->c_thr >= 0.f) || o->randfib < 0 || o->randfib > 3 || o->fibst < 1)
    return api_fail(BPX_ERR_INVALID_ARG, "bpx_probtrack_dev: bad steplength, cthr, randfib or fibst");
  if (v->nx < 1 || v->ny < 1 || v->nz < 1 || v->nfib < 1 || v->nfib > BPX_MAX_FIBRES || v->nsamples < 1)
    return api_fail(BPX_ERR_INVALID_ARG, "bpx_probtrack_dev: bad grid, fibre or sample count");
  if ((size_t)v->nx * v->ny * v->nz >= (1ull << 32))
    return api_fail(BPX_ERR_UNSUPPORTED, "bpx_probtrack_dev: more than 2^32 voxels");
  if ((size_t)v->nx * v->ny * v->nz * (size_t)v->nsamples >= (1ull << 36) || v->nsamples > (1 << 20))
    return api_fail(BPX_ERR_UNSUPPORTED, "bpx_probtrack_dev: more than 2^36 samples, or 2^20 per voxel");
  if (!(v->dx > 0.f && v->dy > 0.f && v->dz > 0.f))
    return api_fail(BPX_ERR_INVALID_ARG, "bpx_probtrack_dev: voxel sizes must be positive");
  if (o->fibst > v->nfib) return api_fail(BPX_ERR_INVALID_ARG, "bpx_probtrack_dev: fibst beyond the fibres given");
  if (nseeds < 0) return api_fail(BPX_ERR_INVALID_ARG, "bpx_probtrack_dev: nseeds < 0");
  if (v->nwaypoints < 0 || v->nwaypoints > 32)
    return api_fail(BPX_ERR_INVALID_ARG, "bpx_probtrack_dev: nwaypoints must be in 0..32");
  if (v->ntargets < 0 || v->ntargets > 32)
    return api_fail(BPX_ERR_INVALID_ARG, "bpx_probtrack_dev: ntargets must be in 0..32");
  if (v->ntargets > 0 && o->pathdist)
    return api_fail(BPX_ERR_UNSUPPORTED, "bpx_probtrack_dev: seeds to targets with pathdist");
  if (nseeds > 0 && v->ntargets > 0 && (!v->targets || !v->seeds_to_targets))
    return api_fail(BPX_ERR_INVALID_ARG, "bpx_probtrack_dev: NULL targets or seeds_to_targets");
  if (v->m2_ncols < 0) return api_fail(BPX_ERR_INVALID_ARG, "bpx_probtrack_dev: m2_ncols < 0");
  if (v->m2_ncols > 0) {
    if (v->lr_nx < 1 || v->lr_ny < 1 || v->lr_nz < 1 || !(v->lr_dx > 0.f && v->lr_dy > 0.f && v->lr_dz > 0.f))
      return api_fail(BPX_ERR_INVALID_ARG, "bpx_probtrack_dev: bad tract-space grid for matrix2");
    if ((size_t)v->nx * v->ny * v->nz >= (1ull << 31) || (size_t)v->lr_nx * v->lr_ny * v->lr_nz >= (1ull << 31))
      return api_fail(BPX_ERR_UNSUPPORTED, "bpx_probtrack_dev: matrix2 with 2^31 or more voxels in either grid");
    if ((size_t)nseeds * (size_t)v->m2_ncols >= (1ull << 40))
      return api_fail(BPX_ERR_UNSUPPORTED, "bpx_probtrack_dev: matrix2 of 2^40 or more entries");
    if (nseeds > 0 && (!v->m2_lookup || !v->matrix2))
      return api_fail(BPX_ERR_INVALID_ARG, "bpx_probtrack_dev: NULL m2_lookup or matrix2");
  }
  if (v->m1_ncols < 0) return api_fail(BPX_ERR_INVALID_ARG, "bpx_probtrack_dev: m1_ncols < 0");
  if (v->m1_ncols > 0) {
    if ((size_t)nseeds * (size_t)v->m1_ncols >= (1ull << 40))
      return api_fail(BPX_ERR_UNSUPPORTED, "bpx_probtrack_dev: matrix1 of 2^40 or more entries");
    if (nseeds > 0 && (!v->m1_lookup || !v->matrix1))
      return api_fail(BPX_ERR_INVALID_ARG, "bpx_probtrack_dev: NULL m1_lookup or matrix1");
  }
  if (nseeds > 0 && (!seeds || !paths || !waytotal || !v->th || !v->ph || !v->f || !v->mask ||
                     (v->nwaypoints > 0 && !v->waypoints)))
    return api_fail(BPX_ERR_INVALID_ARG, "bpx_probtrack_dev: NULL buffer");
  return BPX_OK;
}

}  // namespace
}  // namespace bpx

using namespace bpx;

extern "C" {

void bpx_track_options_default(bpx_track_options* o) {
  if (!o) return;
  *o = bpx_track_options{};
  o->nparticles = 5000;
  o->nsteps = 2000;
  o->steplength = 0.5f;
  o->c_thr = 0.2f;
  o->fibthresh = 0.01f;
  o->distthresh = 0.f;
  o->randfib = 0;
  o->fibst = 1;
  o->seed = 8665904ull;
}

bpx_status bpx_probtrack_dev(const bpx_track_options* opts, const bpx_track_volume* vol, int32_t nseeds,
                             const float* seeds, int32_t* paths, int64_t* waytotal, void* stream) {
  NvtxRange nvtx_range("bpx.probtrack");
  bpx_status st = check_track(opts, vol, nseeds, seeds, paths, waytotal);
  if (st != BPX_OK || nseeds == 0) return st;
  st = api_check_device();
  if (st != BPX_OK) return st;
  TrackArgs a{};
  a.o = *opts;
  a.v = *vol;
  a.nvox = (size_t)vol->nx * vol->ny * vol->nz;
  a.sx = opts->steplength / vol->dx;
  a.sy = opts->steplength / vol->dy;
  a.sz = opts->steplength / vol->dz;
  if (vol->m2_ncols > 0) {
    a.lrx = vol->dx / vol->lr_dx;
    a.lry = vol->dy / vol->lr_dy;
    a.lrz = vol->dz / vol->lr_dz;
  }
  a.nseeds = nseeds;
  a.seeds = seeds;
  a.paths = reinterpret_cast<int*>(paths);
  a.waytotal = reinterpret_cast<unsigned long long*>(waytotal);
  // a table of at least twice the longest path (one voxel per step of both halves, and one
  // tract-space voxel per step with matrix2)
  const long long keys = (long long)(opts->nsteps + 2) * (vol->m2_ncols > 0 ? 2 : 1);
  int log2n = 1;
  while ((1ll << log2n) < 2ll * keys) ++log2n;
  a.log2n = log2n;
  // --loopcheck: a table of at least twice the coarse cells one half can enter.  A half's path is at
  // most l = (nsteps / 2) * steplength / min(dx, dy, dz) voxels long; cut into pieces of at most 4
  // voxels, each piece meets at most 8 cells of 5 voxels, so it enters at most 8 (ceil(l / 4) + 1)
  a.lcnx = vol->nx / 5 + 2;
  a.lcny = vol->ny / 5 + 2;
  const long long lc_cells = (long long)a.lcnx * a.lcny * (vol->nz / 5 + 2);
  const float dmin = fminf(vol->dx, fminf(vol->dy, vol->dz));
  const double half_len = (double)(opts->nsteps / 2) * (double)opts->steplength / (double)dmin;
  const double lc_geom = 8.0 * (std::ceil(half_len / 4.0) + 1.0);
  long long lc_max = lc_cells < opts->nsteps / 2 + 1 ? lc_cells : opts->nsteps / 2 + 1;
  if (lc_geom < (double)lc_max) lc_max = (long long)lc_geom;
  int lc_log2n = 1;
  while ((1ll << lc_log2n) < 2 * lc_max) ++lc_log2n;
  a.lc_log2n = lc_log2n;
  const size_t lc_bytes = opts->loopcheck ? ((size_t)1 << lc_log2n) * (sizeof(uint2) + sizeof(float4)) : 0;
  // particles in flight: kTrackBlocksPerSm blocks per SM, fewer when the tables of very long paths
  // would pass 16 GB
  const size_t table_bytes = ((size_t)1 << log2n) * sizeof(uint2);
  const size_t max_blocks = ((size_t)16 << 30) / ((table_bytes + lc_bytes) * kTrackThreads);
  const int feat = (opts->modeuler ? kFeatEuler : 0) | (opts->loopcheck ? kFeatLoop : 0) |
                   ((vol->ntargets > 0 || vol->m2_ncols > 0 || vol->m1_ncols > 0) ? kFeatCount : 0) |
                   (vol->prefdir ? kFeatPref : 0);
  int grid = sm_count() * kTrackBlocksPerSm;
  if ((size_t)grid > max_blocks) grid = max_blocks > 0 ? (int)max_blocks : 1;
  const size_t threads = (size_t)grid * kTrackThreads;
  // workspace: the visit tables, the loopcheck tables (keys, then directions), the repacked samples
  const int pk4 = vol->nfib + 1;
  const size_t tab_total = (threads * table_bytes + 255) & ~(size_t)255;
  const size_t lc_keys = opts->loopcheck ? (threads * ((size_t)1 << lc_log2n) * sizeof(uint2) + 255) & ~(size_t)255 : 0;
  const size_t lc_dirs = opts->loopcheck ? threads * ((size_t)1 << lc_log2n) * sizeof(float4) : 0;
  const size_t packed_bytes = a.nvox * (size_t)vol->nsamples * (size_t)pk4 * sizeof(float4);
  void* ws = nullptr;
  st = api_workspace(kWsTrack, tab_total + lc_keys + lc_dirs + packed_bytes, &ws);
  if (st != BPX_OK) return st;
  a.tables = (uint2*)ws;
  a.lc_keys = opts->loopcheck ? (uint2*)((char*)ws + tab_total) : nullptr;
  a.lc_dirs = opts->loopcheck ? (float4*)((char*)ws + tab_total + lc_keys) : nullptr;
  a.packed = (const float4*)((char*)ws + tab_total + lc_keys + lc_dirs);
  a.pk4 = pk4;
  cudaStream_t s = (cudaStream_t)stream;
  {
    const dim3 block(kPackTile, 8);
    const dim3 pgrid((unsigned)((a.nvox + kPackTile - 1) / kPackTile), (unsigned)((vol->nsamples + kPackTile - 1) / kPackTile));
    pack_samples_kernel<<<pgrid, block, 0, s>>>(vol->th, vol->ph, vol->f, vol->nfib, vol->nsamples, a.nvox, pk4,
                                                 (float4*)a.packed);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return api_cuda_fail(e, "bpx_probtrack_dev: pack_samples_kernel");
  }
  const uint64_t total = (uint64_t)nseeds * (uint64_t)opts->nparticles;
  const uint64_t chunk = 1ull << 30;  // stamps stay below 2^30 + 1 within a launch
  for (uint64_t b = 0; b < total; b += chunk) {
    // stamp 0 marks every entry empty before a launch reuses the tables
    const cudaError_t e0 = cudaMemsetAsync(ws, 0, tab_total + lc_keys, s);
    if (e0 != cudaSuccess) return api_cuda_fail(e0, "bpx_probtrack_dev: cudaMemsetAsync");
    a.pid_begin = b;
    a.pid_end = b + chunk < total ? b + chunk : total;
    switch (feat) {
      case 0: track_kernel<0><<<grid, kTrackThreads, 0, s>>>(a); break;
      case 1: track_kernel<1><<<grid, kTrackThreads, 0, s>>>(a); break;
      case 2: track_kernel<2><<<grid, kTrackThreads, 0, s>>>(a); break;
      case 3: track_kernel<3><<<grid, kTrackThreads, 0, s>>>(a); break;
      case 4: track_kernel<4><<<grid, kTrackThreads, 0, s>>>(a); break;
      case 5: track_kernel<5><<<grid, kTrackThreads, 0, s>>>(a); break;
      case 6: track_kernel<6><<<grid, kTrackThreads, 0, s>>>(a); break;
      case 7: track_kernel<7><<<grid, kTrackThreads, 0, s>>>(a); break;
      case 8: track_kernel<8><<<grid, kTrackThreads, 0, s>>>(a); break;
      case 9: track_kernel<9><<<grid, kTrackThreads, 0, s>>>(a); break;
      case 10: track_kernel<10><<<grid, kTrackThreads, 0, s>>>(a); break;
      case 11: track_kernel<11><<<grid, kTrackThreads, 0, s>>>(a); break;
      case 12: track_kernel<12><<<grid, kTrackThreads, 0, s>>>(a); break;
      case 13: track_kernel<13><<<grid, kTrackThreads, 0, s>>>(a); break;
      case 14: track_kernel<14><<<grid, kTrackThreads, 0, s>>>(a); break;
      default: track_kernel<15><<<grid, kTrackThreads, 0, s>>>(a); break;
    }
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return api_cuda_fail(e, "bpx_probtrack_dev: track_kernel");
  }
  return BPX_OK;
}

}  // extern "C"
