// sem_kernels.cu — sm_100a kernels and C-ABI runtime for the 2-D acoustic SEM
// forward solver and adjoint gradient of MUN's sem_waveform package.
//
// Discrete algorithm (restated, not translated):
//   Forward step (Bspline_Coupling/SEM/sem_waveform/core.py:598-659, 1197-1211) keeps
//   (u_prev, u_curr) and computes u_next = 2 u_curr - u_prev + dt^2 M^-1 (-K u_curr + f),
//   then multiplies all three by the sponge decay d (boundary.py:5-106) and rotates.
//   Here the state is (b, v) = (u_curr, u_curr - u_prev), which is the same recurrence:
//     w = v - dt^2 M^-1 K b + dt^2 s_t e_src,   v' = d.w,   b' = d.(b + w)
//   but keeps float32 rounding out of the velocity: storing two displacement levels
//   rounds each independently and every rounding acts as a velocity kick amplified by
//   1/(omega dt) (about 10-20x larger seismogram error, measured).
//   Adjoint step (core.py:1252-1275): the same recurrence run backwards with the
//   source R^T r_it / sigma^2, no sponge (or the sponge, in exact mode), and the
//   per-step sensitivity of core.py:49-85 summed over time in float64 (float32 partial
//   sums of at most 16 ticks folded into a float64 field; see kGradFold).
//
// Operator structure used here.  With rectangular affine elements and GLL
// collocation, Gx = (2/dx) kron(L,D), Gz = (2/dz) kron(D,L) with L diagonal
// (operators.py:6-42; L = diag(l) because of the 1e-12 in utils.py:31-37), so the
// element stiffness splits into 1-D operators along grid lines:
//   (K u)[gx,gz] = Rz[gz] * sum_{x-elements e ∋ gx} (D^T (beta c^2 (D u_e)))[i]
//                + Rx[gx] * sum_{z-elements e ∋ gz} (D^T (beta c^2 (D u_e)))[j]
// with beta_a = w_a l_a, Rz[gz] = J (2/dx)^2 sum_{z-elements} w_j l_j^3 and Rx the
// same with x and z swapped; lumped mass and sponge are separable as well.  The same
// split gives the sensitivity  dJ/dc^2 = Rz * sum beta (D u)(D lam) + Rx * (...).
//
// Kernel organisation (owner computes, no atomics): one CTA per tile of elements.
// It stages the tile's node values plus an N-node halo (the neighbour elements'
// nodes) in shared memory, evaluates every element segment that touches an owned
// node (x-lines then z-lines), and writes each owned node once, summing the two
// segment contributions of element-boundary nodes in a fixed order — deterministic
// and bit-reproducible, so the checkpoint replay regenerates the forward exactly.
//
// Time program.  A "tick" advances every active solve of a batch by one action:
// forward step t, one final receiver read-out, checkpoint replay step, or adjoint
// step.  Each CTA decodes its solve's action from (tick - start_tick) with a pure
// function, so a fixed launch sequence (capturable in a CUDA graph) drives any mix
// of solves with different nt, checkpoint interval and polynomial order.

#include <cuda.h>  // CUtensorMap and its encoder's types (the encoder is fetched at run time)
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <type_traits>
#include <vector>

#include "../../include/mun_sem.h"

namespace {

constexpr int kMaxN = 7;       // supported polynomial orders 1..7
// tile kernel: the tick body compiled separately for adjoint and forward-like ticks
#ifndef SEM_TILE_SPLIT
#define SEM_TILE_SPLIT 0
#endif
constexpr int kMaxInj = 1024;  // receivers whose element touches one tile (checked on the host)
constexpr int kInjCache = 8;   // adjoint-source receivers of a tile staged before the tile

// ----------------------------------------------------------------------------
// error plumbing
// ----------------------------------------------------------------------------
thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

#define CUDA_TRY(expr)                                                           \
  do {                                                                           \
    cudaError_t _e = (expr);                                                     \
    if (_e != cudaSuccess) {                                                     \
      return fail(_e == cudaErrorMemoryAllocation ? SEM_ERR_OOM : SEM_ERR_CUDA,  \
                  std::string(#expr) + ": " + cudaGetErrorString(_e));           \
    }                                                                            \
  } while (0)

// ----------------------------------------------------------------------------
// device-side solve descriptor
// ----------------------------------------------------------------------------
enum : int { F_ADJ = SEM_F_ADJOINT, F_EXACT = SEM_F_EXACT, F_MISFIT = SEM_F_MISFIT,
             F_SHIFT = SEM_F_SHIFT };
enum : int { A_NONE = 0, A_FWD = 1, A_FINAL = 2, A_REPLAY = 3, A_ADJ = 4, A_SCALE = 5 };

struct SolveDev {
  // geometry
  int nelx, nelz, nxg, nzg, pitch;
  int tiles_x, tiles_z, tile_base;
  int zchunk;         // strip kernel: element rows per CTA (nelz: full-height strips)
  // program
  int nt, k, nseg, flags, start_tick;
  int it0, it1, decim;
  int src_gx, src_gz;
  int nrec;
  int bnd_n;          // Stacey / free-surface mode: boundary slots (0: the sponge)
  int bnd_pitch;      // floats per row of the boundary tables (bnd_n rounded up to 64)
  long long fstride;  // floats per state field
  // fields
  const float* c2;
  float* W;     // 2 fields: displacement b ping-pong
  float* V;     // 1 field: increment v (updated in place by its owner)
  float* ckpt;  // 2*nseg fields: (b, v) at t = j*k; slots 0,1 = the zero initial state
  float* ring;  // k+1 fields: b at t = j*k .. j*k+k of the segment being replayed
  float* L;     // 2 fields: adjoint lambda ping-pong
  float* Mu;    // 1 field: adjoint increment (in place)
  float* grad;     // 1 field: float32 partial sum of dJ/dc^2 (times the adjoint scale)
                   //   over at most kGradFold adjoint ticks
  double* grad64;  // float64 field (2 float slots): the partial sums folded over time
  // operators and tables
  const float* D;     // (N+1)^2
  const float* beta;  // N+1
  const float* tx;    // 3*nxg
  const float* tz;    // 3*nzg
  const float* src_term;
  // receivers
  const int* rec_base;
  const float* rec_w;
  const int* rec_tile_off;
  const int* rec_tile_ids;
  const int* inj_tile_off;
  const int* inj_tile_ids;
  float* rec_out;
  const double* yobs;
  double* misfit;     // [nrec] sum of squared residuals
  double* rmax;       // [nrec] max |residual| (sizes the adjoint source)
  double* adj_scale;  // [1] power-of-two scale applied to the adjoint source
  int* status;
  // strip kernel: the workspace base (its float fields start at multiples of fstride) and
  // the tensor map of the band loads over it (device memory; null for the tile kernel)
  const float* ws;
  const void* tmap;
  // Stacey mode: per slot e1 = (1 - a) / (1 + a), e2 = 1 / (1 + a) and the impedance-term
  // factor g (rows of bnd_pitch floats), and, for adjoint solves, the boundary nodes' b_t
  // for t = 0 .. nt (row t), written by forward and replay ticks
  const float* bnd_coef;
  float* bnd_hist;
};

__device__ __forceinline__ void decode(const SolveDev& s, int sig, int& act, int& t, int& seg) {
  act = A_NONE;
  t = 0;
  seg = -1;
  if (sig < 0) return;
  if (sig < s.nt) { act = A_FWD; t = sig; return; }
  sig -= s.nt;
  if (s.flags & F_SHIFT) {
    if (sig == 0) { act = A_FINAL; t = s.nt; return; }
    sig -= 1;
  }
  if (!(s.flags & F_ADJ)) return;
  if (sig == 0) { act = A_SCALE; return; }
  sig -= 1;
  const int jl = s.nseg - 1;
  const int len_last = s.nt - jl * s.k;
  if (sig < len_last) { act = A_ADJ; t = s.nt - 1 - sig; seg = jl; return; }
  sig -= len_last;
  if (sig >= 2 * s.k * jl) return;
  const int j = jl - 1 - sig / (2 * s.k);
  const int w = sig % (2 * s.k);
  seg = j;
  if (w < s.k) { act = A_REPLAY; t = j * s.k + w; }
  else { act = A_ADJ; t = (j + 1) * s.k - 1 - (w - s.k); }
}

// Programmatic dependent launch: a tick kernel lets the next tick's grid start launching
// at once (its CTAs run their prologue in this grid's tail) and, before touching any
// field, waits until the previous grid in the stream has completed.  Every CTA waits
// before it may exit, so grid completion stays ordered along the stream.  Both are no-ops
// for a plain launch.
__device__ __forceinline__ void grid_dep_launch() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
__device__ __forceinline__ void grid_dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// where b_t / v_t live during the forward sweep (t in [0, nt])
__device__ __forceinline__ const float* fwd_b(const SolveDev& s, int t) {
  if (!(s.flags & F_ADJ)) return s.W + (long long)(t & 1) * s.fstride;
  const int jl = s.nseg - 1;
  if (t >= jl * s.k) return s.ring + (long long)(t - jl * s.k) * s.fstride;
  if (t % s.k == 0) return s.ckpt + (long long)(2 * (t / s.k)) * s.fstride;
  return s.W + (long long)(t & 1) * s.fstride;
}
__device__ __forceinline__ const float* fwd_v(const SolveDev& s, int t) {
  if (!(s.flags & F_ADJ)) return s.V;
  const int jl = s.nseg - 1;
  if (t < jl * s.k && t % s.k == 0) return s.ckpt + (long long)(2 * (t / s.k) + 1) * s.fstride;
  return s.V;
}
// where b_t / v_t live while segment j is replayed (t in [jk, jk+k])
__device__ __forceinline__ const float* rep_b(const SolveDev& s, int j, int t) {
  if (t == j * s.k) return s.ckpt + (long long)(2 * j) * s.fstride;
  return s.ring + (long long)(t - j * s.k) * s.fstride;
}
__device__ __forceinline__ const float* rep_v(const SolveDev& s, int j, int t) {
  if (t == j * s.k) return s.ckpt + (long long)(2 * j + 1) * s.fstride;
  return s.V;
}

__host__ __device__ __forceinline__ int region_w(int tex, int N) { return ((tex + 2) * N + 1) | 1; }
__host__ __device__ __forceinline__ int region_h(int tez, int N) { return (tez + 2) * N + 1; }

// shared-memory floats needed by one CTA
__host__ __device__ inline long long smem_floats(int N, int tex, int tez, bool adj) {
  const int NP = N + 1;
  const long long reg = (long long)region_w(tex, N) * region_h(tez, N);
  const long long nro = (long long)(tez * N + 1) | 1, nco = (long long)(tex * N + 1) | 1;
  const long long xseg = (long long)(tex + 1) * NP * nro, zseg = (long long)(tez + 1) * NP * nco;
  long long f = 96 + 2 * reg + xseg + zseg;  // D, beta | u, c2 | K_x, K_z
  if (adj) f += reg + xseg + zseg + nro * nco + kMaxInj;  // forward field | S_x, S_z | injection
  if (adj) f += kInjCache * (3 + 64);  // first receivers: id, element base, weights
  return f;
}


// The zero-lag sensitivity increment of one node, R_z S_x + R_x S_z, rounded the same way
// in every kernel.
__device__ __forceinline__ float sens_increment(float Rzv, float SX, float Rxv, float SZ) {
  return __fmaf_rn(Rzv, SX, __fmul_rn(Rxv, SZ));
}
// Time-sum of the gradient: the increments of at most kGradFold consecutive adjoint ticks
// are added in a float32 partial sum (one __fadd_rn per node and tick), which is folded
// into the float64 accumulator on the ticks with (t - it0) % kGradFold == 0 (__dadd_rn);
// the last gradient tick, t = it0, is one of them.  A partial starts from zero on the
// tick after a fold and on the first gradient tick (t = it1 - 1), so it is never read
// there.  Per node and adjoint tick that moves 8 bytes plus a 16-byte float64
// read-modify-write every kGradFold ticks, and adds a few 1e-8 relative error against
// float64 accumulation of the same increments.
constexpr int kGradFold = 16;
__device__ __forceinline__ bool grad_partial_starts(const SolveDev& s, int t) {
  return t == s.it1 - 1 || (t - s.it0) % kGradFold == kGradFold - 1;
}
__device__ __forceinline__ bool grad_folds(const SolveDev& s, int t) { return (t - s.it0) % kGradFold == 0; }
// Sensitivity of one segment node, beta_a (D w)_a (D lambda)_a, multiplied left to right.
__device__ __forceinline__ float sens_product(float beta, float dw, float du) {
  return __fmul_rn(__fmul_rn(beta, dw), du);
}

// One receiver's read-out sum_e w_e u_e computed by one thread with the roundings of the
// one-warp form the tile kernel uses: lane l sums terms l, l + 32, ... by FMA from zero,
// then the lanes are combined by the xor-shuffle tree (offsets 16, 8, 4, 2, 1), whose
// value on lane 0 is the pairwise tree below.  u_e is b[(e / NP) * bw + e % NP].
template <int N>
__device__ __forceinline__ float rec_dot_tree(const float* __restrict__ wr, const float* b, int bw) {
  constexpr int NP = N + 1, NE = NP * NP;
  float v[32];
#pragma unroll
  for (int l = 0; l < 32; ++l) {
    float a = 0.f;
#pragma unroll
    for (int e = l; e < NE; e += 32) a = fmaf(__ldg(wr + e), b[(e / NP) * bw + (e % NP)], a);
    v[l] = a;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
    for (int l = 0; l < o; ++l) v[l] = __fadd_rn(v[l], v[l + o]);
  }
  return v[0];
}

// One owned node: combine the line operators, advance (b, v) or (lambda, mu), apply
// the sponge.  Shared by both kernel variants so their arithmetic is identical.
//   forward:  w = v - P K + src          adjoint: w = mu + P (inj - K)
//   v' = d w, b' = d (b + w)   (d = 1 in the reference-mode adjoint), with d = 1 - delta
//   applied as w - delta w and s - delta s (dxv, dzv: the tables' decay defects)
__device__ __forceinline__ void advance_node(bool adj, bool damp, float b, float v, float X,
                                             float Z, float ixv, float Rxv, float dxv, float izv,
                                             float Rzv, float dzv, float extra, float& bout,
                                             float& vout) {
  // explicit rounding: the same operations in every kernel that inlines this, whatever
  // the compiler would contract
  const float P = __fmul_rn(ixv, izv);
  const float Kv = __fmaf_rn(Rzv, X, __fmul_rn(Rxv, Z));
  float wv;
  if (!adj) {
    wv = __fadd_rn(__fmaf_rn(-P, Kv, v), extra);
  } else {
    wv = __fmaf_rn(P, __fsub_rn(extra, Kv), v);
  }
  if (damp) {
    // sponge: the decay d = (1 - dx)(1 - dz) applied as s - delta s, delta = 1 - d from the
    // tables' defects (a float32 decay just below 1 would be a fixed bias every step)
    const float dl = __fmaf_rn(-dxv, dzv, __fadd_rn(dxv, dzv));
    vout = __fmaf_rn(-dl, wv, wv);
    const float s = __fadd_rn(b, wv);
    bout = __fmaf_rn(-dl, s, s);
  } else {
    vout = wv;
    bout = __fadd_rn(b, wv);
  }
}

// Stacey / free-surface mode (an extension; the reference has only the sponge).  Slot of a
// node of the absorbing edges (x = xmin, x = xmax, z = zmax) in the boundary tables, or -1.
__device__ __forceinline__ int bnd_slot(const SolveDev& s, int gx, int gz) {
  if (gx == 0) return gz;
  if (gx == s.nxg - 1) return s.nzg + gz;
  if (gz == s.nzg - 1) return 2 * s.nzg + gx;
  return -1;
}
// One node in the Stacey mode: (1 + a) u+ = 2 u - (1 - a) u- + F in the (b, v) state,
//   w = e1 v + e2 F,  v' = w,  b' = b + w   (e1 = (1 - a) / (1 + a), e2 = 1 / (1 + a) on the
// absorbing edges, e1 = e2 = 1 elsewhere), F = extra - P K (forward) or P (extra - K)
// (adjoint, the same recurrence run backwards); there is no sponge in this mode.  Every
// node of a Stacey solve takes this form in both kernels.
__device__ __forceinline__ void advance_node_stacey(bool adj, float b, float v, float X, float Z,
                                                    float ixv, float Rxv, float izv, float Rzv,
                                                    float extra, float e1, float e2, float& bout,
                                                    float& vout) {
  const float P = __fmul_rn(ixv, izv);
  const float Kv = __fmaf_rn(Rzv, X, __fmul_rn(Rxv, Z));
  const float F = !adj ? __fmaf_rn(-P, Kv, extra) : __fmul_rn(P, __fsub_rn(extra, Kv));
  const float w = __fmaf_rn(e1, v, __fmul_rn(e2, F));
  vout = w;
  bout = __fadd_rn(b, w);
}
// The gradient's boundary-impedance increment (from d a / d c) of slot k at adjoint tick
// t <= nt - 2, added to the sensitivity of c^2:  g lambda (b_{t+2} - b_t).
__device__ __forceinline__ float bnd_sens(const SolveDev& s, int k, int t, float lam) {
  const long long BP = s.bnd_pitch;
  const float du = __fsub_rn(s.bnd_hist[(long long)(t + 2) * BP + k], s.bnd_hist[(long long)t * BP + k]);
  return __fmul_rn(__fmul_rn(s.bnd_coef[2 * BP + k], lam), du);
}

// ----------------------------------------------------------------------------
// tile kernel: one CTA per tile of elements (used for small batches)
// ----------------------------------------------------------------------------
// Loads of data that other CTAs of the same launch may have written: in the persistent
// kernel (one launch for every tick, grid barrier between ticks) they bypass L1, which
// is not coherent across SMs; the per-tick kernels read through the read-only path.
template <bool COH>
__device__ __forceinline__ float ld_xf(const float* p) {
  if constexpr (COH) return __ldcg(p); else return __ldg(p);
}
template <bool COH>
__device__ __forceinline__ double ld_xd(const double* p) {
  if constexpr (COH) return __ldcg(p); else return *p;
}

// One tick of one element tile (act != A_NONE), shared by the per-tick tile kernel and
// the persistent kernel (COH: cross-CTA data read coherently).
// SPLIT: compiled for one tick kind, ADJ (adjoint ticks) or not (forward, read-out, scale);
// without SPLIT one body decides at run time (same arithmetic either way)
template <int N, bool COH, bool SPLIT = false, bool ADJ = false>
__device__ __forceinline__ void tile_tick(const SolveDev& S, const int act, const int t,
                                          const int seg, const int tex, const int tez,
                                          float* smem) {
  constexpr int NP = N + 1;
  const bool adj = SPLIT ? ADJ : (act == A_ADJ);
  if (act == A_SCALE) {
    // one CTA per solve picks the power of two that brings max|r| to ~1, so the
    // float32 adjoint field and the sensitivity products stay far from underflow
    if (blockIdx.x == S.tile_base && threadIdx.x == 0) {
      double m = 0.0;
      for (int r = 0; r < S.nrec; ++r) m = fmax(m, ld_xd<COH>(S.rmax + r));
      *S.adj_scale = (m > 0.0 && isfinite(m)) ? ldexp(1.0, -ilogb(m)) : 1.0;
    }
    return;
  }

  // ---------------- tile geometry
  const int lt = blockIdx.x - S.tile_base;
  const int tx = lt % S.tiles_x, tz = lt / S.tiles_x;
  const int ex0 = tx * tex, ex1 = min(ex0 + tex, S.nelx);
  const int ez0 = tz * tez, ez1 = min(ez0 + tez, S.nelz);
  const int gxo0 = ex0 * N, gxo1 = (ex1 == S.nelx) ? S.nxg : ex1 * N;
  const int gzo0 = ez0 * N, gzo1 = (ez1 == S.nelz) ? S.nzg : ez1 * N;
  const int nco = gxo1 - gxo0, nro = gzo1 - gzo0;
  const int gxs = gxo0 - N, gzs = gzo0 - N;
  const int SW = region_w(tex, N), SH = region_h(tez, N);
  const int segx0 = max(ex0 - 1, 0), nsx = ex1 - segx0;
  const int segz0 = max(ez0 - 1, 0), nsz = ez1 - segz0;
  const int nrop = nro | 1, ncop = nco | 1;
  const int REG = SW * SH;
  const int nrop_max = (tez * N + 1) | 1, ncop_max = (tex * N + 1) | 1;

  float* sD = smem;
  float* sB = smem + 64;
  float* su = smem + 96;                 // current field (b_t or lambda)
  float* sc = su + REG;                  // c^2
  float* sw = sc + REG;                  // forward field for the sensitivity (adjoint)
  float* xr = sw + (adj ? REG : 0);
  float* zr = xr + (tex + 1) * NP * nrop_max;
  float* xs = zr + (tez + 1) * NP * ncop_max;
  float* zs = xs + (tex + 1) * NP * nrop_max;
  float* sacc = zs + (tez + 1) * NP * ncop_max;

  const int nthr = blockDim.x;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = nthr >> 5;

  // ---------------- which fields (b: read with halo; v: read/written by the owner only)
  const float* cur;
  const float* vin = nullptr;
  float* out = nullptr;
  float* vout = nullptr;
  const float* fwdu = nullptr;
  if (act == A_FWD) {
    cur = fwd_b(S, t); vin = fwd_v(S, t);
    out = (float*)fwd_b(S, t + 1); vout = (float*)fwd_v(S, t + 1);
  } else if (act == A_FINAL) {
    cur = fwd_b(S, t);
  } else if (act == A_REPLAY) {
    cur = rep_b(S, seg, t); vin = rep_v(S, seg, t);
    out = (float*)rep_b(S, seg, t + 1); vout = (float*)rep_v(S, seg, t + 1);
  } else {  // adjoint iteration it = t: lambda_{t+1} -> lambda_t, forward b_{t+1}
    cur = S.L + (long long)((t + 1) & 1) * S.fstride;
    out = S.L + (long long)(t & 1) * S.fstride;
    vin = S.Mu;
    vout = S.Mu;
    fwdu = S.ring + (long long)(t + 1 - seg * S.k) * S.fstride;
  }

  // ---------------- this thread's first owned node: its own inputs are loaded before the
  // tile is staged, so their latency overlaps the staging (small tiles are latency-bound)
  const int w0 = threadIdx.x;
  const bool pre = (act != A_FINAL) && w0 < nro * nco;
  float p_v = 0.f, p_ix = 0.f, p_Rx = 0.f, p_dx = 0.f, p_iz = 0.f, p_Rz = 0.f, p_dz = 0.f;
  float p_g = 0.f;
  if (pre) {
    const int gx = gxo0 + w0 % nco, gz = gzo0 + w0 / nco;
    const long long g0 = (long long)gz * S.pitch + gx;
    p_v = vin[g0];
    p_ix = __ldg(S.tx + gx); p_Rx = __ldg(S.tx + S.nxg + gx); p_dx = __ldg(S.tx + 2 * S.nxg + gx);
    p_iz = __ldg(S.tz + gz); p_Rz = __ldg(S.tz + S.nzg + gz); p_dz = __ldg(S.tz + 2 * S.nzg + gz);
    if (adj && t >= S.it0 && t < S.it1 && !grad_partial_starts(S, t)) p_g = S.grad[g0];
  }
  // the same for the misfit terms of each warp's first receiver (forward ticks)
  const int rec_m = t - ((S.flags & F_SHIFT) ? 1 : 0);
  const bool rec_tick = (act == A_FWD || act == A_FINAL) && rec_m >= 0 && rec_m < S.nt;
  const bool mis_tick = rec_tick && (S.flags & F_MISFIT) && rec_m >= S.it0 && rec_m < S.it1 &&
                        ((rec_m - S.it0) % S.decim) == 0;
  // and of this thread's first adjoint-source receiver (adjoint ticks in the window)
  const bool in_win = adj && t >= S.it0 && t < S.it1 && ((t - S.it0) % S.decim) == 0;
  float p_res = 0.f;
  if (in_win && (int)threadIdx.x < S.inj_tile_off[lt + 1] - S.inj_tile_off[lt]) {
    const int r = S.inj_tile_ids[S.inj_tile_off[lt] + threadIdx.x];
    const long long yrow = (long long)((t - S.it0) / S.decim) * S.nrec;
    const double res = (double)ld_xf<COH>(S.rec_out + (long long)t * S.nrec + r) - S.yobs[yrow + r];
    p_res = (float)(res * ld_xd<COH>(S.adj_scale));
  }
  // the first receivers' ids, element bases and weights: a warp's first read-out receiver
  // in registers, the first kInjCache adjoint-source receivers in shared memory
  int* const s_ir = reinterpret_cast<int*>(sacc + nrop_max * ncop_max + kMaxInj);
  int* const s_ibx = s_ir + kInjCache;
  int* const s_ibz = s_ibx + kInjCache;
  float* const s_iw = reinterpret_cast<float*>(s_ibz + kInjCache);
  if (in_win) {
    const int ioff = S.inj_tile_off[lt], icnt = min(S.inj_tile_off[lt + 1] - ioff, kInjCache);
    if ((int)threadIdx.x < icnt) {
      const int r = S.inj_tile_ids[ioff + threadIdx.x];
      s_ir[threadIdx.x] = r;
      s_ibx[threadIdx.x] = S.rec_base[2 * r];
      s_ibz[threadIdx.x] = S.rec_base[2 * r + 1];
    }
    for (int k = threadIdx.x; k < icnt * NP * NP; k += nthr) {
      const int q = k / (NP * NP), e = k - q * (NP * NP);
      s_iw[q * 64 + e] = S.rec_w[(long long)S.inj_tile_ids[ioff + q] * NP * NP + e];
    }
  }
  const bool rec_first = rec_tick && warp < S.rec_tile_off[lt + 1] - S.rec_tile_off[lt];
  int p_r = 0, p_bx = 0, p_bz = 0;
  float p_w0 = 0.f, p_w1 = 0.f;
  if (rec_first) {
    p_r = S.rec_tile_ids[S.rec_tile_off[lt] + warp];
    p_bx = S.rec_base[2 * p_r];
    p_bz = S.rec_base[2 * p_r + 1];
    const float* wr = S.rec_w + (long long)p_r * NP * NP;
    if (lane < NP * NP) p_w0 = wr[lane];
    if (lane + 32 < NP * NP) p_w1 = wr[lane + 32];
  }
  double p_y = 0.0, p_mis = 0.0, p_rmax = 0.0;
  if (mis_tick && lane == 0 && rec_first) {
    p_y = S.yobs[(long long)((rec_m - S.it0) / S.decim) * S.nrec + p_r];
    p_mis = S.misfit[p_r];
    p_rmax = S.rmax[p_r];
  }

  // ---------------- stage operators and the haloed tile (one (row, column) item per
  // thread and pass: a small tile's halo region takes a single pass)
  for (int i = threadIdx.x; i < NP * NP; i += nthr) sD[i] = S.D[i];
  for (int i = threadIdx.x; i < NP; i += nthr) sB[i] = S.beta[i];
  {
    const int r0 = max(gzs, 0), r1 = min(gzs + SH, S.nzg);
    const int c0 = max(gxs, 0), c1 = min(gxs + (ex1 - ex0 + 2) * N + 1, S.nxg);
    const bool need_c = (act != A_FINAL);
    const int ncol = c1 - c0, tot = ncol * (r1 - r0);
#pragma unroll 2
    for (int i = threadIdx.x; i < tot; i += nthr) {
      const int rr = i / ncol, r = r0 + rr, c = c0 + (i - rr * ncol);
      const long long gi = (long long)r * S.pitch + c;
      const int si = (r - gzs) * SW + (c - gxs);
      su[si] = ld_xf<COH>(cur + gi);
      if (need_c) sc[si] = __ldg(S.c2 + gi);
      if (adj) sw[si] = ld_xf<COH>(fwdu + gi);
    }
  }
  __syncthreads();

  // ---------------- receivers: record R b_t (forward sweep only)
  if (act == A_FWD || act == A_FINAL) {
    const int m = rec_m;
    if (rec_tick) {
      const int off = S.rec_tile_off[lt], cnt = S.rec_tile_off[lt + 1] - off;
      for (int q = warp; q < cnt; q += nwarps) {
        const bool pf = (q == warp);
        const int r = pf ? p_r : S.rec_tile_ids[off + q];
        const int bx = pf ? p_bx : S.rec_base[2 * r], bz = pf ? p_bz : S.rec_base[2 * r + 1];
        const float* wr = S.rec_w + (long long)r * NP * NP;
        float acc = 0.f;
        for (int e = lane; e < NP * NP; e += 32) {
          const int j = e / NP, i = e - j * NP;
          const float we = !pf ? wr[e] : (e < 32 ? p_w0 : p_w1);
          acc = fmaf(we, su[(bz + j - gzs) * SW + (bx + i - gxs)], acc);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) {
          S.rec_out[(long long)m * S.nrec + r] = acc;
          if (mis_tick) {
            const bool first = (q == warp);
            const double res =
                (double)acc - (first ? p_y : S.yobs[(long long)((m - S.it0) / S.decim) * S.nrec + r]);
            S.misfit[r] = __dadd_rn(first ? p_mis : S.misfit[r], __dmul_rn(res, res));
            S.rmax[r] = fmax(first ? p_rmax : S.rmax[r], fabs(res));
          }
        }
      }
    }
    if (act == A_FINAL) return;
  }

  // ---------------- adjoint source R^T r_it: residuals of this tile's receivers are
  // formed in parallel, then one warp adds them node by node in receiver order
  // (deterministic; receivers of one element never race)
  bool have_inj = false;
  if (adj) {
    const int off = S.inj_tile_off[lt], cnt = S.inj_tile_off[lt + 1] - off;
    have_inj = in_win && cnt > 0;
    if (have_inj) {
      float* sres = sacc + nrop_max * ncop_max;  // cnt <= kMaxInj floats
      const double ascale = ld_xd<COH>(S.adj_scale);
      const long long yrow = (long long)((t - S.it0) / S.decim) * S.nrec;
      for (int i = threadIdx.x; i < nro * nco; i += nthr) sacc[i] = 0.f;
      for (int q = threadIdx.x; q < cnt; q += nthr) {
        if (q == (int)threadIdx.x) {
          sres[q] = p_res;
          continue;
        }
        const int r = S.inj_tile_ids[off + q];
        const double res = (double)ld_xf<COH>(S.rec_out + (long long)t * S.nrec + r) - S.yobs[yrow + r];
        sres[q] = (float)(res * ascale);
      }
      __syncthreads();
      if (warp == 0) {
        for (int q = 0; q < cnt; ++q) {
          const bool cached = q < kInjCache;
          const int r = cached ? s_ir[q] : S.inj_tile_ids[off + q];
          const float rs = sres[q];
          const int bx = cached ? s_ibx[q] : S.rec_base[2 * r];
          const int bz = cached ? s_ibz[q] : S.rec_base[2 * r + 1];
          const float* wr = S.rec_w + (long long)r * NP * NP;
          for (int e = lane; e < NP * NP; e += 32) {
            const int j = e / NP, i = e - j * NP;
            const int gx = bx + i, gz = bz + j;
            const float we = cached ? s_iw[q * 64 + e] : wr[e];
            if (gx >= gxo0 && gx < gxo1 && gz >= gzo0 && gz < gzo1)
              sacc[(gz - gzo0) * nco + (gx - gxo0)] =
                  __fmaf_rn(we, rs, sacc[(gz - gzo0) * nco + (gx - gxo0)]);
          }
          __syncwarp();
        }
      }
    }
  }

  // ---------------- x-lines: one thread per (owned row, element segment)
  for (int w = threadIdx.x; w < nro * nsx; w += nthr) {
    const int r = w % nro, sg = w / nro;
    const int ex = segx0 + sg;
    const int base = (gzo0 + r - gzs) * SW + (ex * N - gxs);
    float u[NP], c[NP], du[NP], q[NP];
#pragma unroll
    for (int a = 0; a < NP; ++a) { u[a] = su[base + a]; c[a] = sc[base + a]; }
#pragma unroll
    for (int a = 0; a < NP; ++a) {
      float v = 0.f;
#pragma unroll
      for (int b = 0; b < NP; ++b) v = fmaf(sD[a * NP + b], u[b], v);
      du[a] = v;
      q[a] = sB[a] * c[a] * v;
    }
#pragma unroll
    for (int i = 0; i < NP; ++i) {
      float v = 0.f;
#pragma unroll
      for (int a = 0; a < NP; ++a) v = fmaf(sD[a * NP + i], q[a], v);
      xr[(sg * NP + i) * nrop + r] = v;
    }
    if (adj) {
#pragma unroll
      for (int a = 0; a < NP; ++a) u[a] = sw[base + a];
#pragma unroll
      for (int a = 0; a < NP; ++a) {
        float v = 0.f;
#pragma unroll
        for (int b = 0; b < NP; ++b) v = fmaf(sD[a * NP + b], u[b], v);
        xs[(sg * NP + a) * nrop + r] = sens_product(sB[a], v, du[a]);
      }
    }
  }
  // ---------------- z-lines: one thread per (owned column, element segment)
  for (int w = threadIdx.x; w < nco * nsz; w += nthr) {
    const int cc = w % nco, sg = w / nco;
    const int ez = segz0 + sg;
    const int base = (ez * N - gzs) * SW + (gxo0 + cc - gxs);
    float u[NP], c[NP], du[NP], q[NP];
#pragma unroll
    for (int a = 0; a < NP; ++a) { u[a] = su[base + a * SW]; c[a] = sc[base + a * SW]; }
#pragma unroll
    for (int a = 0; a < NP; ++a) {
      float v = 0.f;
#pragma unroll
      for (int b = 0; b < NP; ++b) v = fmaf(sD[a * NP + b], u[b], v);
      du[a] = v;
      q[a] = sB[a] * c[a] * v;
    }
#pragma unroll
    for (int j = 0; j < NP; ++j) {
      float v = 0.f;
#pragma unroll
      for (int a = 0; a < NP; ++a) v = fmaf(sD[a * NP + j], q[a], v);
      zr[(sg * NP + j) * ncop + cc] = v;
    }
    if (adj) {
#pragma unroll
      for (int a = 0; a < NP; ++a) u[a] = sw[base + a * SW];
#pragma unroll
      for (int a = 0; a < NP; ++a) {
        float v = 0.f;
#pragma unroll
        for (int b = 0; b < NP; ++b) v = fmaf(sD[a * NP + b], u[b], v);
        zs[(sg * NP + a) * ncop + cc] = sens_product(sB[a], v, du[a]);
      }
    }
  }
  __syncthreads();

  // ---------------- owned nodes: assemble, Newmark, sponge, source / sensitivity
  const bool damp = (act != A_ADJ) || (S.flags & F_EXACT);
  const bool grad_on = adj && t >= S.it0 && t < S.it1;
  const bool g_start = grad_on && grad_partial_starts(S, t);
  const bool g_fold = grad_on && grad_folds(S, t);
  const bool stc = S.bnd_n > 0;
  bool bad = false;
  for (int w = threadIdx.x; w < nro * nco; w += nthr) {
    const int cc = w % nco, r = w / nco;
    const int gx = gxo0 + cc, gz = gzo0 + r;
    const int exr = gx / N, ia = gx - exr * N;
    const int ezr = gz / N, ja = gz - ezr * N;
    float X, Z, SX = 0.f, SZ = 0.f;
    if (ia) {
      const int o = ((exr - segx0) * NP + ia) * nrop + r;
      X = xr[o];
      if (adj) SX = xs[o];
    } else {
      X = 0.f;
      if (exr >= 1) {
        const int o = ((exr - 1 - segx0) * NP + N) * nrop + r;
        X = xr[o];
        if (adj) SX = xs[o];
      }
      if (exr < S.nelx) {
        const int o = ((exr - segx0) * NP) * nrop + r;
        X = __fadd_rn(X, xr[o]);
        if (adj) SX = __fadd_rn(SX, xs[o]);
      }
    }
    if (ja) {
      const int o = ((ezr - segz0) * NP + ja) * ncop + cc;
      Z = zr[o];
      if (adj) SZ = zs[o];
    } else {
      Z = 0.f;
      if (ezr >= 1) {
        const int o = ((ezr - 1 - segz0) * NP + N) * ncop + cc;
        Z = zr[o];
        if (adj) SZ = zs[o];
      }
      if (ezr < S.nelz) {
        const int o = ((ezr - segz0) * NP) * ncop + cc;
        Z = __fadd_rn(Z, zr[o]);
        if (adj) SZ = __fadd_rn(SZ, zs[o]);
      }
    }
    const bool first = (w == w0);
    const float ixv = first ? p_ix : __ldg(S.tx + gx), Rxv = first ? p_Rx : __ldg(S.tx + S.nxg + gx);
    const float izv = first ? p_iz : __ldg(S.tz + gz), Rzv = first ? p_Rz : __ldg(S.tz + S.nzg + gz);
    const float dxv = first ? p_dx : __ldg(S.tx + 2 * S.nxg + gx);
    const float dzv = first ? p_dz : __ldg(S.tz + 2 * S.nzg + gz);
    const long long g = (long long)gz * S.pitch + gx;
    const float b = su[(gz - gzs) * SW + (gx - gxs)];
    const float v = first ? p_v : vin[g];
    const int bk = (stc && gz > 0) ? bnd_slot(S, gx, gz) : -1;
    float extra = 0.f;
    if (!adj) {
      if (gx == S.src_gx && gz == S.src_gz) extra = S.src_term[t];
    } else {
      extra = have_inj ? sacc[r * nco + cc] : 0.f;
      if (grad_on) {
        const float gprev = g_start ? 0.f : (first ? p_g : S.grad[g]);
        float inc = sens_increment(Rzv, SX, Rxv, SZ);
        if (bk >= 0 && t <= S.nt - 2) inc = __fadd_rn(inc, bnd_sens(S, bk, t, b));
        const float gnew = __fadd_rn(gprev, inc);
        if (g_fold)
          S.grad64[g] = __dadd_rn(S.grad64[g], (double)gnew);
        else
          S.grad[g] = gnew;
      }
    }
    float res, vres;
    if (stc) {
      // Stacey mode: w = e1 v + e2 F at every node, e1 = e2 = 1 off the absorbing edges
      // (the strip kernel's form, so both give the same bits); u = 0 on the free surface
      const long long BP = S.bnd_pitch;
      const float e1 = bk >= 0 ? S.bnd_coef[bk] : 1.f, e2 = bk >= 0 ? S.bnd_coef[BP + bk] : 1.f;
      advance_node_stacey(adj, b, v, X, Z, ixv, Rxv, izv, Rzv, extra, e1, e2, res, vres);
      if (gz == 0) {
        res = 0.f;
        vres = 0.f;
      }
      if (bk >= 0 && !adj && (S.flags & F_ADJ)) S.bnd_hist[(long long)(t + 1) * BP + bk] = res;
    } else {
      advance_node(adj, damp, b, v, X, Z, ixv, Rxv, dxv, izv, Rzv, dzv, extra, res, vres);
    }
    vout[g] = vres;
    out[g] = res;
    bad |= !isfinite(res);
  }
  if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(S.status, SEM_ERR_NONFINITE);
}

template <int N>
__global__ void __launch_bounds__(256) sem_tick_kernel(const SolveDev* __restrict__ solves,
                                                       const int* __restrict__ cta_solve,
                                                       const int* __restrict__ tick_ptr,
                                                       int tex, int tez, int tick_arg) {
  extern __shared__ float smem[];
  __shared__ SolveDev S;
  __shared__ int s_act, s_t, s_seg;
  grid_dep_launch();

  const int sid = cta_solve[blockIdx.x];
  {
    static_assert(sizeof(SolveDev) % 8 == 0, "descriptor is copied as 8-byte words");
    const unsigned long long* src = reinterpret_cast<const unsigned long long*>(solves + sid);
    unsigned long long* dst = reinterpret_cast<unsigned long long*>(&S);
    for (int i = threadIdx.x; i < (int)(sizeof(SolveDev) / 8); i += blockDim.x) dst[i] = src[i];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int act, t, seg;
    decode(S, (tick_ptr ? *tick_ptr : tick_arg) - S.start_tick, act, t, seg);
    s_act = act; s_t = t; s_seg = seg;
  }
  __syncthreads();
  grid_dep_wait();  // the previous tick's fields are complete from here on
  const int act = s_act;
  if (act == A_NONE) return;
#if SEM_TILE_SPLIT
  if (act == A_ADJ)
    tile_tick<N, false, true, true>(S, act, s_t, s_seg, tex, tez, smem);
  else
    tile_tick<N, false, true, false>(S, act, s_t, s_seg, tex, tez, smem);
#else
  tile_tick<N, false>(S, act, s_t, s_seg, tex, tez, smem);
#endif
}

// ----------------------------------------------------------------------------
// strip kernel: one CTA per full-height strip of element columns (large batches)
//
// Columns: N left-halo columns, the strip's owned columns and the shared column on its
// right.  The CTA sweeps the strip one element row ("band", N+1 grid rows) at a time;
// the band of every field the step reads is staged by TMA tensor copies (cp.async.bulk.tensor +
// mbarrier; one box per field from a tiled tensor map over the solve's workspace) into a
// ring of 3 slots, issued as many bands ahead as there are slots.
// Work per band: one thread per (band row, element segment) for the x-lines, one thread
// per owned column for the z-line segment of the band, D and beta in registers; then
// one thread per owned column combines the segment results and advances the band's
// nodes.  Arithmetic order matches the tile kernel (bitwise-equal results).
// ----------------------------------------------------------------------------
#ifndef SEM_PDL
#define SEM_PDL 1
#endif
#ifndef SEM_PAIRED
#define SEM_PAIRED 1
#endif
#ifndef SEM_STAGES_ADJ
#define SEM_STAGES_ADJ 3
#endif
// Stacey edge values a band ahead: 0 = register staging by 50 carrier threads,
// 1 = cp.async copies
#ifndef SEM_BND_ASYNC
#define SEM_BND_ASYNC 0
#endif
// adjoint ticks: D (lambda) and D (forward field) of a segment in packed FFMA2
#ifndef SEM_PAIRED_ADJ
#define SEM_PAIRED_ADJ 1
#endif
#ifndef SEM_STRIP_MIN_BLOCKS
#define SEM_STRIP_MIN_BLOCKS 4
#endif
// suspend-time hint of the ring waits (ns); 0 = the instruction's own short suspend window,
// measured 1-2 % faster per tick than a 20 us hint (the wait stays bounded either way)
#ifndef SEM_WAIT_HINT_NS
#define SEM_WAIT_HINT_NS 0
#endif
constexpr int kStripCols = 128;
constexpr int kStages = 3;                   // ring slots of forward/replay ticks
constexpr int kStagesAdj = SEM_STAGES_ADJ;   // ring slots of adjoint ticks (bigger bands)
constexpr int kStripInj = 256;               // receivers per band of one strip (host-checked)
constexpr int kMapBands = 8;                 // strip chunks this tall load bands by tensor map
constexpr long long kWaitNs = 2000000000LL;  // bounded mbarrier waits: 2 s
// floats ahead of the ring: mbarriers (64), D (64), beta (16), the band's z-table rows (48)
constexpr int kStripHdr = 192;
// The strip kernel's operator constants: the GLL derivative matrix D and the factors beta
// depend only on the order, so each device keeps one copy per order in constant memory
// (filled at plan creation); FMAs take them as uniform constant operands, which keeps 30
// registers free for the band's work.
__constant__ float c_D[kMaxN + 1][64];
__constant__ float c_B[kMaxN + 1][8];
// the same values duplicated into both halves of a float2, for packed FFMA2 / FMUL2
__constant__ float2 c_D2[kMaxN + 1][64];
__constant__ float2 c_B2[kMaxN + 1][8];

__host__ __device__ inline int strip_ew_max(int N) { return (kStripCols - N - 1) / N; }
__host__ __device__ inline int strip_bw(int /*N*/) { return (kStripCols + 3 + 3) & ~3; }  // smem row
__host__ __device__ inline int strip_threads(int /*N*/) { return kStripCols; }

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
#if SEM_BND_ASYNC
// 4-byte asynchronous global -> shared copies (the Stacey edge values, a band ahead)
__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
#endif
__device__ __forceinline__ void mbar_inval(unsigned long long* bar) {
  asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
#if SEM_WAIT_HINT_NS > 0
  // suspend until the phase completes (or the hint elapses) instead of spinning
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity), "r"((unsigned)SEM_WAIT_HINT_NS)
      : "memory");
#else
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
#endif
  return ok != 0;
}
__device__ __forceinline__ long long global_ns() {
  long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// wait for a TMA phase; gives up after kWaitNs and reports false
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = global_ns();
  while (!mbar_try_wait(bar, parity))
    if (global_ns() - t0 > kWaitNs) return false;
  return true;
}

// floats of one staged field of a band (N+1 rows of strip_bw columns), rounded up so that
// every field's block starts 128-byte aligned (tensor-copy destinations)
__host__ __device__ inline int strip_field_floats(int N) { return ((N + 1) * strip_bw(N) + 31) & ~31; }
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes,
                                          unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}
// one box of a 3-D tiled tensor map (column x, row y, field slot z) into shared memory;
// x is a multiple of 4 floats (16 bytes), negative or past the edge reads zeros
__device__ __forceinline__ void tensor_load_3d(void* dst, const void* tmap, int x, int y, int z,
                                               unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
      ::"r"(smem_addr(dst)), "l"(tmap), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
      : "memory");
}
// the map was written by the host through the generic proxy: make it visible to the
// tensor-copy proxy before its first use in this launch
__device__ __forceinline__ void tensormap_acquire(const void* tmap) {
  asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(tmap) : "memory");
}

__host__ __device__ inline long long strip_stage_floats(int N, bool adj) {
  const int nfloat = adj ? 4 : 3;  // cur, c2, v (+ forward field); the gradient is
                                   // loaded by its owner threads, not staged
  return (long long)nfloat * strip_field_floats(N);
}
// exchange arrays: x-segment results Xs[rows][segments][N+1] (+ sensitivity), z-segment
// results stay in registers; injection rows and residuals
__host__ __device__ inline long long strip_xch_floats(int N, bool adj) {
  const long long NP = N + 1, segs = strip_ew_max(N) + 1;
  const long long nb = 2;                                            // exchange buffers
  long long f = nb * (adj ? 2 : 1) * NP * segs * NP;                 // Xs | SXs (per buffer)
  if (adj) f += NP * kStripCols + kStripInj;                         // inj | res
  return (f + 31) & ~31LL;
}
constexpr int kStripBndSide = 3 * 2 * 5 * 8;                   // Stacey edge values by band
constexpr int kStripBndFloats = kStripBndSide + 5 * kStripCols;  // + the bottom row
__host__ __device__ inline long long strip_smem_floats(int N, bool adj) {
  const long long fwd = kStages * strip_stage_floats(N, false) + strip_xch_floats(N, false);
  const long long adjf = kStagesAdj * strip_stage_floats(N, true) + strip_xch_floats(N, true);
  return kStripHdr + (adj ? (fwd > adjf ? fwd : adjf) : fwd);
}

// Loads the N+1 consecutive floats of one x-line segment.  For N = 4 the strip's copy
// origin puts every element edge on a 4-float boundary: one float4, and the shared edge
// node comes from the next lane's first value when that lane holds the next segment of
// the same row (`from_next`), else from shared memory.
template <int N>
__device__ __forceinline__ void load_seg(const float* p, float (&u)[N + 1], unsigned mask,
                                         bool from_next) {
  if constexpr (N == 4) {
    const float4 q = *reinterpret_cast<const float4*>(p);
    u[0] = q.x; u[1] = q.y; u[2] = q.z; u[3] = q.w;
    const float nx = __shfl_down_sync(mask, q.x, 1);
    u[4] = from_next ? nx : p[4];
  } else {
#pragma unroll
    for (int b = 0; b <= N; ++b) u[b] = p[b];
  }
}

// Paired phase A: every lane loads its x-line segment (zeros when it has no item) so
// that the whole warp takes part in the edge-node shuffle.
template <int N>
__device__ __forceinline__ void load_seg_all(const float* p, bool valid, bool from_next,
                                             float (&u)[N + 1]) {
  if constexpr (N == 4) {
    const float4 q = valid ? *reinterpret_cast<const float4*>(p) : make_float4(0.f, 0.f, 0.f, 0.f);
    u[0] = q.x; u[1] = q.y; u[2] = q.z; u[3] = q.w;
    const float nx = __shfl_down_sync(0xffffffffu, q.x, 1);
    u[4] = from_next ? nx : (valid ? p[4] : 0.f);
  } else {
#pragma unroll
    for (int b = 0; b <= N; ++b) u[b] = valid ? p[b] : 0.f;
  }
}

// Receivers read out of one band of a strip, one thread each (the sum as rec_dot_tree,
// bitwise the tile kernel's one-warp form), with their misfit terms.  Out of line: the
// band loop's register allocation does not carry this block, which runs in few bands.
template <int N>
__device__ __noinline__ void strip_read_out(const SolveDev& S, const float* Bs, int X0, int r0, int cnt,
                                            int ms) {
  constexpr int NP = N + 1;
  constexpr int BW = (kStripCols + 3 + 3) & ~3;
  const bool mis = (S.flags & F_MISFIT) && ms >= S.it0 && ms < S.it1 && ((ms - S.it0) % S.decim) == 0;
  for (int q = threadIdx.x; q < cnt; q += kStripCols) {
    const int r = S.rec_tile_ids[r0 + q];
    // the misfit terms are fetched before the sum so that their loads overlap it
    double y = 0.0, m0 = 0.0, rm0 = 0.0;
    if (mis) {
      y = S.yobs[(long long)((ms - S.it0) / S.decim) * S.nrec + r];
      m0 = S.misfit[r];
      rm0 = S.rmax[r];
    }
    const float acc = rec_dot_tree<N>(S.rec_w + (long long)r * NP * NP, Bs + (S.rec_base[2 * r] - X0), BW);
    S.rec_out[(long long)ms * S.nrec + r] = acc;
    if (mis) {
      const double res = (double)acc - y;
      S.misfit[r] = __dadd_rn(m0, __dmul_rn(res, res));
      S.rmax[r] = fmax(rm0, fabs(res));
    }
  }
}

// Adjoint source of the receivers of one band of a strip (adjoint ticks in the misfit
// window): residuals one thread each, then the weights and element bases of up to kw
// receivers at a time in scr (an exchange buffer that phase A of the band does not write;
// phase B of the previous band, its last reader, is behind the first barrier below), and
// each owned column adds the terms of the receivers whose element holds it, in receiver
// order: per node the same FMAs in the same order as one warp walking the receivers.
// Every thread of the CTA calls it (it holds barriers).  Out of line as strip_read_out.
template <int N, bool COH>
__device__ __noinline__ void strip_inject(const SolveDev& S, int t, int j0, int cnt, float* sacc, float* sres,
                                          float* scr, int kw_max, bool owned, int gx) {
  constexpr int NP = N + 1, NE = NP * NP, NT = kStripCols;
  const int tid = threadIdx.x;
  // (COH: written by other CTAs of this launch, read past L1)
  const double ascale = COH ? __ldcg(S.adj_scale) : *S.adj_scale;
  const long long yrow = (long long)((t - S.it0) / S.decim) * S.nrec;
  for (int q = tid; q < cnt; q += NT) {
    const int r = S.inj_tile_ids[j0 + q];
    const float* rp = S.rec_out + (long long)t * S.nrec + r;
    const double res = (double)(COH ? __ldcg(rp) : *rp) - S.yobs[yrow + r];
    sres[q] = (float)(res * ascale);
  }
  int* const sbx = reinterpret_cast<int*>(scr + kw_max * NE);
  float iacc[NP];
#pragma unroll
  for (int j = 0; j < NP; ++j) iacc[j] = owned ? sacc[j * NT + tid] : 0.f;
  for (int c0 = 0; c0 < cnt; c0 += kw_max) {
    const int kw = min(kw_max, cnt - c0);
    __syncthreads();
    for (int k = tid; k < kw * NE; k += NT) {
      const int q = k / NE;
      scr[k] = S.rec_w[(long long)S.inj_tile_ids[j0 + c0 + q] * NE + (k - q * NE)];
    }
    for (int q = tid; q < kw; q += NT) sbx[q] = S.rec_base[2 * S.inj_tile_ids[j0 + c0 + q]];
    __syncthreads();
    if (owned) {
      for (int q = 0; q < kw; ++q) {
        const int i = gx - sbx[q];
        if (i >= 0 && i <= N) {
          const float rs = sres[c0 + q];
#pragma unroll
          for (int j = 0; j < NP; ++j) iacc[j] = __fmaf_rn(scr[q * NE + j * NP + i], rs, iacc[j]);
        }
      }
    }
  }
  if (owned) {
#pragma unroll
    for (int j = 0; j < NP; ++j) sacc[j * NT + tid] = iacc[j];
  }
}

// One tick of one strip chunk (element rows [zb0, zb1) of one strip), instantiated for
// forward-like ticks (FWD, FINAL, REPLAY) and for adjoint ticks so that neither carries
// the other's branches.  A chunk below the first starts with a halo band (element row
// zb0 - 1): only its z-line segments (the carry into row zb0 * N) and its adjoint
// injection carry are computed there; the chunk above owns that band.
template <int N, bool ADJ, bool COH, bool STC>
__device__ __forceinline__ void strip_tick(const SolveDev& S, const int act, const int t,
                                           const int seg, float* smem, int* s_abort) {
  constexpr int NP = N + 1;
  constexpr int BW = (kStripCols + 3 + 3) & ~3;
  constexpr int NT = kStripCols;
  constexpr int NW = NT / 32;
  constexpr int SEGS = (kStripCols - N - 1) / N + 1;  // x-segments per band row (max)
  constexpr int NF = ADJ ? 4 : 3;                      // staged float fields
  constexpr int NST = ADJ ? kStagesAdj : kStages;      // ring slots
  constexpr int XSZ = (ADJ ? 2 : 1) * NP * SEGS * NP;  // floats of one exchange buffer
  const bool final_only = !ADJ && act == A_FINAL;

  // ---------------- strip geometry (tiles_z = elements per strip)
  const int nelx = S.nelx, nelz = S.nelz, nxg = S.nxg, nzg = S.nzg, pitch = S.pitch;
  const int zch = S.zchunk > 0 ? S.zchunk : nelz;          // element rows per chunk
  const int nzc = (nelz + zch - 1) / zch;                   // chunks per strip
  const int local = blockIdx.x - S.tile_base;
  const int strip = local / nzc, chunk = local - strip * nzc;
  const int zb0 = chunk * zch, zb1 = min(nelz, zb0 + zch);  // owned element rows
  const bool has_halo = zb0 > 0 && !final_only;
  const int ezs = zb0 - (has_halo ? 1 : 0);                 // first band processed
  const int nbands = zb1 - ezs;
  const int EW = S.tiles_z;
  const int e0 = strip * EW, e1 = min(e0 + EW, nelx);
  const int sx0 = e0 * N;                                   // first owned column
  const int so1 = (e1 == nelx) ? nxg : e1 * N;              // owned columns [sx0, so1)
  const int X0 = (sx0 - N) & ~3;                            // 16-byte aligned copy origin
  const int off = (sx0 - N) - X0;                           // smem column of column sx0 - N
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nseg = e1 - e0 + 1;                             // segments e0-1 .. e1-1
  const int seg0 = (e0 == 0) ? 1 : 0;                       // segment -1 does not exist
  const int gx = sx0 + tid;                                 // this thread's owned column
  const bool owned = gx < so1;
  const int sc = tid + N + off;                             // its smem column

  // ---------------- shared memory
  unsigned long long* bars = reinterpret_cast<unsigned long long*>(smem);
  float* const sTz = smem + 64 + 64 + 16;         // [2][3][8] band rows of 1/mz, Rz, dz
  const long long stage_f = strip_stage_floats(N, ADJ);
  float* const stages = smem + kStripHdr;
  float* const xs0 = stages + NST * stage_f;      // 2 exchange buffers: Xs [NP][SEGS][NP] (+ SXs)
  float* const sacc = xs0 + 2 * XSZ;              // adjoint: injection rows [NP][NT]
  float* const sres = sacc + NP * NT;             // adjoint: band residuals [kStripInj]
  // Stacey mode: the edge values of a band (e1, e2, g, b_t, b_{t+2}) for the left and right
  // columns, 3 buffers by band, and of the bottom row, behind the tick kind's own layout
  float* const sbnd = smem + strip_smem_floats(N, ADJ);  // [3][2 sides][5][8]
  float* const bbot = sbnd + kStripBndSide;              // [5][NT]

  // ---------------- which fields
  const float* cur;
  const float* vin = nullptr;
  float* out = nullptr;
  float* vout = nullptr;
  const float* fwdu = nullptr;
  if (ADJ) {
    cur = S.L + (long long)((t + 1) & 1) * S.fstride;
    out = S.L + (long long)(t & 1) * S.fstride;
    vin = S.Mu;
    vout = S.Mu;
    fwdu = S.ring + (long long)(t + 1 - seg * S.k) * S.fstride;
  } else if (act == A_FWD) {
    cur = fwd_b(S, t); vin = fwd_v(S, t);
    out = (float*)fwd_b(S, t + 1); vout = (float*)fwd_v(S, t + 1);
  } else if (act == A_FINAL) {
    cur = fwd_b(S, t);
  } else {
    cur = rep_b(S, seg, t); vin = rep_v(S, seg, t);
    out = (float*)rep_b(S, seg, t + 1); vout = (float*)rep_v(S, seg, t + 1);
  }
  const float* const c2p = S.c2;
  float* const gradp = S.grad;
  const float* const tzp = S.tz;
  const int nload = final_only ? 1 : NF;

  if (tid == 0) {
    for (int s2 = 0; s2 < NST; ++s2) mbar_init(bars + s2, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  // TMA: element row `ez` of every field into ring slot (ez - ezs) % NST; thread 0 posts
  // the expected bytes (a copy may complete first: the barrier's pending arrival keeps
  // the phase open until then).  Field f of a band lands in the slot's block f.
  //  * chunks of at least kMapBands bands: one tensor copy per field, the box of BW
  //    columns from X0 and N+1 rows from ez * N of the field's slot in the solve's
  //    workspace map (columns outside [0, pitch) read as zeros and are never used),
  //    issued by lane 1 of warp f.  Fewer, larger copies; the map's acquire and first
  //    fetch cost a little per CTA and tick, which short chunks do not amortise.
  //  * shorter chunks: one bulk copy per (field, row), spread over all warps (copy
  //    q = lane * NW + warp), each thread fixing its source and destination once per tick.
  constexpr int FBF = ((N + 1) * BW + 31) & ~31;  // floats per staged field block
  const bool by_map = S.tmap != nullptr && nbands >= kMapBands;
  const int cs = max(X0, 0), ce = min(X0 + BW, pitch);  // columns inside the field
  const unsigned rowb = (unsigned)(ce - cs) * 4u;
  const int myq = by_map ? (lane == 1 && warp < nload ? warp : NT) : lane * NW + warp;
  const bool has_copy = by_map ? myq < nload : myq < nload * NP;
  int cp_dst = 0, cp_slot = 0;
  const float* cp_src = cur;
  if (has_copy) {
    const int f = by_map ? myq : myq / NP, a = by_map ? 0 : myq - f * NP;
    const float* fp = (f == 0) ? cur : (f == 1) ? c2p : (f == 2) ? vin : fwdu;
    if (by_map) {
      cp_slot = (int)((fp - S.ws) / S.fstride);
      cp_dst = f * FBF;
      tensormap_acquire(S.tmap);
    } else {
      cp_src = fp + (long long)a * pitch + cs;
      cp_dst = f * FBF + a * BW + (cs - X0);
    }
  }
  const long long band_floats = (long long)N * pitch;
  const unsigned band_bytes = by_map ? (unsigned)(nload * NP * BW) * 4u : (unsigned)(nload * NP) * rowb;
  auto issue = [&](int ez) {
    const int slot = (ez - ezs) % NST;
    if (tid == 0) mbar_expect_tx(bars + slot, band_bytes);
    if (has_copy) {
      if (by_map)
        tensor_load_3d(stages + slot * stage_f + cp_dst, S.tmap, X0, ez * N, cp_slot, bars + slot);
      else
        bulk_load(stages + slot * stage_f + cp_dst, cp_src + ez * band_floats, rowb, bars + slot);
    }
  };
  for (int r = 0; r < min(NST, nbands); ++r) issue(ezs + r);

  // Stacey mode: this CTA's edges (strip 0 owns column 0, the last strip column nxg - 1,
  // the last chunk row nzg - 1) and the asynchronous fetch of their values one band ahead
  const bool side_l = STC && sx0 == 0;
  const bool side_r = STC && so1 == nxg;
  const bool side_col = STC && owned && (gx == 0 || gx == nxg - 1);  // this thread's column
  const bool bottom = STC && zb1 == nelz && !final_only;
  const bool bgterm = ADJ && t >= S.it0 && t < S.it1 && t <= S.nt - 2;  // impedance term
  // the value thread tid < 50 carries: side sd, quantity q (e1, e2, g, b_t, b_{t+2}), row a
  const int bsd = tid / (5 * NP), bq = (tid / NP) % 5, ba = tid % NP;
  const bool bcarrier = STC && tid < 2 * 5 * NP && (bsd == 0 ? side_l : side_r) && (bq < 2 || bgterm);
  auto bnd_src = [&](int ez) -> const float* {
    const int gz = ez * N + ba;
    if (!bcarrier || gz <= 0 || gz >= nzg) return nullptr;
    const long long k = (bsd == 0 ? 0 : nzg) + gz, BP = S.bnd_pitch;
    return bq < 3 ? S.bnd_coef + bq * BP + k : S.bnd_hist + (bq == 3 ? t : t + 2) * BP + k;
  };
#if SEM_BND_ASYNC
  auto bnd_fetch = [&](int ez, int buf) {
    const float* src = bnd_src(ez);
    if (src) cp_async4(sbnd + ((buf * 2 + bsd) * 5 + bq) * 8 + ba, src);
  };
#else
  float bnd_next = 0.f;  // this carrier's value for the next band, loaded a band ahead
#endif
  if (STC) {
    if (bottom && gx > 0 && gx < nxg - 1 && owned) {
      const long long k = 2 * nzg + gx, BP = S.bnd_pitch;
      for (int q = 0; q < (bgterm ? 5 : 2); ++q) {
        const float* src = q < 3 ? S.bnd_coef + q * BP + k : S.bnd_hist + (q == 3 ? t : t + 2) * BP + k;
#if SEM_BND_ASYNC
        cp_async4(bbot + q * NT + tid, src);
#else
        bbot[q * NT + tid] = *src;  // once per tick, before the first band
#endif
      }
    }
#if SEM_BND_ASYNC
    if (!final_only) bnd_fetch(ezs, 0);
#else
    if (!final_only && bnd_src(ezs)) bnd_next = *bnd_src(ezs);
#endif
  }

  // D and beta: per-order constants (c_D[N], c_B[N])
#define Dr(a, b) c_D[N][(a) * NP + (b)]
#define Bt(a) c_B[N][(a)]
  float ixv = 0.f, Rxv = 0.f, dxv = 0.f;
  if (owned) { ixv = __ldg(S.tx + gx); Rxv = __ldg(S.tx + nxg + gx); dxv = __ldg(S.tx + 2 * nxg + gx); }
  // this column's x-segment results: its element's segment at local index ia, or on an
  // element edge the left segment's last and the right segment's first entries
  const int e_r = gx / N, ia = gx - e_r * N;
  const int s_r = e_r - e0 + 1;
  const bool edge = (ia == 0);
  const bool hasL = edge && e_r >= 1;
  const bool hasR = !edge || e_r < nelx;
  const int xoR = s_r * NP + ia;
  const int xoL = (s_r - 1) * NP + N;
  // x-line items: rows 0..N-1 of each band as (row tid / nseg, segment tid % nseg), which
  // fits one item per thread; row N of the last band by threads tid < nseg.  The next
  // lane holds the next segment of the same row when its item is valid and sgi + 1 < nseg.
  const int xa = tid / nseg, xsg = tid - xa * nseg;
  const bool xitem = (xa < N) && (xsg >= seg0);
  const bool xitem_last = (tid < nseg) && (tid >= seg0);
  const unsigned mA = __ballot_sync(0xffffffffu, xitem);
  const unsigned mL = __ballot_sync(0xffffffffu, xitem_last);
  const bool nextA = lane < 31 && ((mA >> (lane + 1)) & 1u) && xsg + 1 < nseg;
  const bool nextL = lane < 31 && ((mL >> (lane + 1)) & 1u) && tid + 1 < nseg;

  const bool damp = !ADJ || (S.flags & F_EXACT);
  const bool grad_on = ADJ && t >= S.it0 && t < S.it1;
  const bool g_start = grad_on && grad_partial_starts(S, t);
  const bool g_fold = grad_on && grad_folds(S, t);
  double* const grad64p = S.grad64;
  // Stacey / free-surface mode (STC) is compiled out of the sponge path
  const bool in_win = ADJ && t >= S.it0 && t < S.it1 && ((t - S.it0) % S.decim) == 0;
  const int ms = t - ((S.flags & F_SHIFT) ? 1 : 0);
  const bool rec_on = !ADJ && (act == A_FWD || act == A_FINAL) && ms >= 0 && ms < S.nt;
  // the source column's thread adds the source term on the source row
  const int src_row = (!ADJ && !final_only && owned && gx == S.src_gx) ? S.src_gz : -1;
  const float src_val = (src_row >= 0) ? S.src_term[t] : 0.f;
  if (ADJ && in_win)
    for (int i = tid; i < NP * NT; i += NT) sacc[i] = 0.f;
  // receiver / injection list bounds of the current band, fetched one band ahead
  const int li0 = strip * nelz;
  int rec_lo = 0, rec_hi = 0, inj_lo = 0, inj_hi = 0;
  if (rec_on) { rec_lo = S.rec_tile_off[li0 + ezs]; rec_hi = S.rec_tile_off[li0 + ezs + 1]; }
  if (ADJ && in_win) { inj_lo = S.inj_tile_off[li0 + ezs]; inj_hi = S.inj_tile_off[li0 + ezs + 1]; }
  // z-table rows: threads tid < 3 NP stage entry (tk, ta) of each band, fetched a band ahead
  const bool tz_thr = !final_only && tid < 3 * NP;
  const int tk = tid / NP, ta = tid - tk * NP;
  float tz_next = tz_thr ? __ldg(tzp + tk * nzg + ezs * N + ta) : 0.f;

  float zc = 0.f, szc = 0.f;  // z-line carries into the next band's first row
  bool bad = false;
  int abort_ez = -1;
  int gb = gx + ezs * N * pitch;  // offset of (row ez * N, column gx) in a field

  for (int rel = 0; rel < nbands; ++rel, gb += N * pitch) {
    const int ez = ezs + rel;      // rel: band index within this chunk's ring sequence
    const int slot = rel % NST;
    const bool halo = has_halo && rel == 0;
    const float* st = stages + slot * stage_f;
    const float* Bs = st;
    const float* Cs = st + FBF;
    const float* Vs = st + 2 * FBF;
    const float* Us = st + 3 * FBF;
    float* const Xs = xs0 + (ez & 1) * XSZ;
    float* const SXs = Xs + NP * SEGS * NP;
    float* const tzb = sTz + (ez & 1) * 24;
    const int r0 = rec_lo, r1 = rec_hi, j0 = inj_lo, j1 = inj_hi;
    if (rel + 1 < nbands) {
      if (rec_on) { rec_lo = rec_hi; rec_hi = S.rec_tile_off[li0 + ez + 2]; }
      if (ADJ && in_win) { inj_lo = inj_hi; inj_hi = S.inj_tile_off[li0 + ez + 2]; }
    }
    if (tz_thr) {
      tzb[tk * 8 + ta] = tz_next;
      if (rel + 1 < nbands) tz_next = __ldg(tzp + tk * nzg + (ez + 1) * N + ta);
    }
    // a failed wait records the first band that failed; every thread tests "failed at or
    // before this band" after the band's barrier, so all threads leave at the same band
    // the owner's gradient rows of this band, loaded now and used in phase B
    float gpre[N];
    if (ADJ && grad_on && !g_start && owned && !halo) {
#pragma unroll
      for (int a = 0; a < N; ++a) gpre[a] = gradp[gb + a * pitch];
    }
    if (STC && !final_only) {
#if SEM_BND_ASYNC
      // this band's edge values (fetched a band ago) are complete once each issuing thread
      // has waited for its copies; the phase-A barrier publishes them.  The next band's go
      // to the buffer no thread reads now (phase B of band rel - 1 reads (rel - 1) % 3).
      cp_async_wait_all();
      if (rel + 1 < nbands) bnd_fetch(ez + 1, (rel + 1) % 3);
#else
      // each carrier parks this band's value (loaded a band ago) for the phase-A barrier to
      // publish, and loads the next band's; phase B of band rel - 1 reads (rel - 1) % 3
      if (bcarrier) {
        sbnd[(((rel % 3) * 2 + bsd) * 5 + bq) * 8 + ba] = bnd_next;
        const float* nsrc = rel + 1 < nbands ? bnd_src(ez + 1) : nullptr;
        if (nsrc) bnd_next = *nsrc;
      }
#endif
    }
    if (!mbar_wait(bars + slot, (unsigned)((rel / NST) & 1))) atomicMin(s_abort, ez);
    const bool last = (ez == nelz - 1);

    if (rec_on && !halo && r1 > r0) strip_read_out<N>(S, Bs, X0, r0, r1 - r0, ms);
    if (final_only) {
      __syncthreads();  // done with this slot
      if (*s_abort <= ez) { abort_ez = ez; break; }
      if (rel + NST < nbands) issue(ez + NST);
      continue;
    }
    if (ADJ && in_win && j1 > j0)  // adjoint source of receivers in this element row
      strip_inject<N, COH>(S, t, j0, j1 - j0, sacc, sres, xs0 + ((ez + 1) & 1) * XSZ,
                           XSZ / (NP * NP + 1), owned, gx);
    // ---- phase A, x-lines: one thread per (band row, element segment)
    auto xline = [&](int a, int sgi, unsigned m, bool nxt) {
      const int o = a * BW + off + sgi * N;  // column (e0 - 1 + sgi) * N of row a
      if constexpr (ADJ && SEM_PAIRED_ADJ) {
        // adjoint ticks: D (lambda) and D (forward field) of the segment as the two halves
        // of packed FFMA2 (per half the scalar fmaf sequence: bitwise the same)
        float u[NP], w[NP], c[NP], q[NP];
        float2 d2[NP];
        load_seg<N>(Bs + o, u, m, nxt);
        load_seg<N>(Us + o, w, m, nxt);
        load_seg<N>(Cs + o, c, m, nxt);
#pragma unroll
        for (int a2 = 0; a2 < NP; ++a2) {
          float2 v = make_float2(0.f, 0.f);
#pragma unroll
          for (int b = 0; b < NP; ++b) v = __ffma2_rn(c_D2[N][a2 * NP + b], make_float2(u[b], w[b]), v);
          d2[a2] = v;
          q[a2] = Bt(a2) * c[a2] * v.x;
        }
        float* xo = Xs + (a * SEGS + sgi) * NP;
#pragma unroll
        for (int i = 0; i < NP; ++i) {
          float v = 0.f;
#pragma unroll
          for (int a2 = 0; a2 < NP; ++a2) v = fmaf(Dr(a2, i), q[a2], v);
          xo[i] = v;
        }
        float* so = SXs + (a * SEGS + sgi) * NP;
#pragma unroll
        for (int a2 = 0; a2 < NP; ++a2) so[a2] = sens_product(Bt(a2), d2[a2].y, d2[a2].x);
        return;
      }
      float u[NP], c[NP], du[NP], q[NP];
      load_seg<N>(Bs + o, u, m, nxt);
      load_seg<N>(Cs + o, c, m, nxt);
#pragma unroll
      for (int a2 = 0; a2 < NP; ++a2) {
        float v = 0.f;
#pragma unroll
        for (int b = 0; b < NP; ++b) v = fmaf(Dr(a2, b), u[b], v);
        du[a2] = v;
        q[a2] = Bt(a2) * c[a2] * v;
      }
      float* xo = Xs + (a * SEGS + sgi) * NP;
#pragma unroll
      for (int i = 0; i < NP; ++i) {
        float v = 0.f;
#pragma unroll
        for (int a2 = 0; a2 < NP; ++a2) v = fmaf(Dr(a2, i), q[a2], v);
        xo[i] = v;
      }
      if (ADJ) {
        load_seg<N>(Us + o, u, m, nxt);
        float* so = SXs + (a * SEGS + sgi) * NP;
#pragma unroll
        for (int a2 = 0; a2 < NP; ++a2) {
          float v = 0.f;
#pragma unroll
          for (int b = 0; b < NP; ++b) v = fmaf(Dr(a2, b), u[b], v);
          so[a2] = sens_product(Bt(a2), v, du[a2]);
        }
      }
    };
    float rz[NP], sz[NP];
    // ---- phase A of forward-like ticks, paired: this thread's x-line segment (lane .x of
    // every float2) and its column's z-line segment (lane .y) share D and beta, so each
    // packed FFMA2 / FMUL2 does one step of both; per half it is the scalar fmaf / multiply
    // sequence.  Adjoint ticks (two more contractions, more live values) stay scalar.
    if (SEM_PAIRED && !ADJ) {
      const bool xi = !halo && xitem;
      const int o = xi ? xa * BW + off + xsg * N : 0;
      float2 u2[NP], c2v[NP], du2[NP], q2[NP];
      {
        float ux[NP], cx[NP];
        load_seg_all<N>(Bs + o, xi, nextA, ux);
        load_seg_all<N>(Cs + o, xi, nextA, cx);
#pragma unroll
        for (int b = 0; b < NP; ++b) {
          u2[b] = make_float2(ux[b], Bs[b * BW + sc]);
          c2v[b] = make_float2(cx[b], Cs[b * BW + sc]);
        }
      }
#pragma unroll
      for (int a2 = 0; a2 < NP; ++a2) {
        float2 v = make_float2(0.f, 0.f);
#pragma unroll
        for (int b = 0; b < NP; ++b) v = __ffma2_rn(c_D2[N][a2 * NP + b], u2[b], v);
        du2[a2] = v;
        q2[a2] = __fmul2_rn(__fmul2_rn(c_B2[N][a2], c2v[a2]), v);
      }
      float* xo = Xs + (xa * SEGS + xsg) * NP;
#pragma unroll
      for (int i = 0; i < NP; ++i) {
        float2 v = make_float2(0.f, 0.f);
#pragma unroll
        for (int a2 = 0; a2 < NP; ++a2) v = __ffma2_rn(c_D2[N][a2 * NP + i], q2[a2], v);
        if (xi) xo[i] = v.x;
        rz[i] = v.y;
      }
      if (!halo && last && xitem_last) xline(N, tid, mL, nextL);
    } else {
      if (!halo) {
        if (xitem) xline(xa, xsg, mA, nextA);
        if (last && xitem_last) xline(N, tid, mL, nextL);
      }
      // ---- phase A, z-lines: one thread per owned column (the band is the segment)
      if (ADJ && SEM_PAIRED_ADJ && owned) {
        float q[NP];
        float2 u2[NP], d2[NP];
#pragma unroll
        for (int b = 0; b < NP; ++b) u2[b] = make_float2(Bs[b * BW + sc], Us[b * BW + sc]);
#pragma unroll
        for (int a2 = 0; a2 < NP; ++a2) {
          float2 v = make_float2(0.f, 0.f);
#pragma unroll
          for (int b = 0; b < NP; ++b) v = __ffma2_rn(c_D2[N][a2 * NP + b], u2[b], v);
          d2[a2] = v;
          q[a2] = Bt(a2) * Cs[a2 * BW + sc] * v.x;
        }
#pragma unroll
        for (int j = 0; j < NP; ++j) {
          float v = 0.f;
#pragma unroll
          for (int a2 = 0; a2 < NP; ++a2) v = fmaf(Dr(a2, j), q[a2], v);
          rz[j] = v;
        }
#pragma unroll
        for (int a2 = 0; a2 < NP; ++a2) sz[a2] = sens_product(Bt(a2), d2[a2].y, d2[a2].x);
      } else if (owned) {
        float u[NP], du[NP], q[NP];
#pragma unroll
        for (int b = 0; b < NP; ++b) u[b] = Bs[b * BW + sc];
#pragma unroll
        for (int a2 = 0; a2 < NP; ++a2) {
          float v = 0.f;
#pragma unroll
          for (int b = 0; b < NP; ++b) v = fmaf(Dr(a2, b), u[b], v);
          du[a2] = v;
          q[a2] = Bt(a2) * Cs[a2 * BW + sc] * v;
        }
#pragma unroll
        for (int j = 0; j < NP; ++j) {
          float v = 0.f;
#pragma unroll
          for (int a2 = 0; a2 < NP; ++a2) v = fmaf(Dr(a2, j), q[a2], v);
          rz[j] = v;
        }
        if (ADJ) {
#pragma unroll
          for (int b = 0; b < NP; ++b) u[b] = Us[b * BW + sc];
#pragma unroll
          for (int a2 = 0; a2 < NP; ++a2) {
            float v = 0.f;
#pragma unroll
            for (int b = 0; b < NP; ++b) v = fmaf(Dr(a2, b), u[b], v);
            sz[a2] = sens_product(Bt(a2), v, du[a2]);
          }
        }
      }
    }
    __syncthreads();
    if (*s_abort <= ez) { abort_ez = ez; break; }
    // every thread is past phase B of the previous band: warp 0 refills its slot
    if (rel >= 1 && rel - 1 + NST < nbands) issue(ez - 1 + NST);
    if (halo) {  // carries into the first owned row only
      if (owned) {
        zc = rz[N];
        if (ADJ) szc = sz[N];
        if (ADJ && in_win) {
          const float carry = sacc[N * NT + tid];
#pragma unroll
          for (int a = 1; a < NP; ++a) sacc[a * NT + tid] = 0.f;
          sacc[tid] = carry;
        }
      }
      continue;
    }
    // ---- phase B: combine and advance the owned nodes of the band, row by row (EDGE:
    // the Stacey mode's copy, compiled out of the sponge path)
    auto phase_b = [&](auto edge_c) {
      constexpr bool EDGE = decltype(edge_c)::value;
      // this band's edge values of this thread's column (Stacey mode): its side column's
      // row of the band buffer, or the bottom row's
      const float* const bv0 = side_col ? sbnd + (((rel % 3) * 2 + (gx == 0 ? 0 : 1)) * 5) * 8 : bbot + tid;
      const int qs = side_col ? 8 : NT;
      // fold ticks: the band's float64 gradient rows, loaded before the first store of the
      // band (issued after those stores they would wait one after another)
      double g64[NP];
      if (ADJ && g_fold) {
#pragma unroll
        for (int a = 0; a < NP; ++a) g64[a] = (a < N || last) ? grad64p[gb + a * pitch] : 0.0;
      }
#pragma unroll
      for (int a = 0; a < NP; ++a) {
        if (a == N && !last) break;
        const float* xr = Xs + a * SEGS * NP;
        const float* sxr = SXs + a * SEGS * NP;
        // interior column: its segment's entry; edge column: left + right (or one of them)
        const float xL = hasL ? xr[xoL] : 0.f;
        const float xR = hasR ? xr[xoR] : 0.f;
        const float X = !edge ? xR : (hasR ? __fadd_rn(xL, xR) : xL);
        float SX = 0.f;
        if (ADJ) {
          const float sL = hasL ? sxr[xoL] : 0.f;
          const float sR = hasR ? sxr[xoR] : 0.f;
          SX = !edge ? sR : (hasR ? __fadd_rn(sL, sR) : sL);
        }
        float Z, SZ = 0.f;
        if (a == 0) {
          // explicit adds: the lower segment's value is computed in this thread and must
          // not be fused with its product into an FMA (the tile kernel adds stored values)
          Z = __fadd_rn(ez >= 1 ? zc : 0.f, rz[0]);
          if (ADJ) SZ = __fadd_rn(ez >= 1 ? szc : 0.f, sz[0]);
        } else {
          Z = rz[a];
          if (ADJ) SZ = sz[a];
        }
        const float izv = tzb[a], Rzv = tzb[8 + a], dzv = tzb[16 + a];
        const int g = gb + a * pitch;
        const int gz = ez * N + a;
        // Stacey mode: the free surface is row 0; the absorbing edges are the side columns
        // (fixed per thread) and the bottom row (row N of the last band)
        const bool top_row = EDGE && ez == 0 && a == 0;
        const bool edge_node = EDGE && !top_row && (side_col || (last && a == N));
        const int bk = !edge_node ? -1 : (gx == 0 ? gz : gx == nxg - 1 ? nzg + gz : 2 * nzg + gx);
        float extra;
        float gnew = 0.f;
        if (!ADJ) {
          extra = (gz == src_row) ? src_val : 0.f;
        } else {
          extra = in_win ? sacc[a * NT + tid] : 0.f;
          if (grad_on) {
            const float gprev = g_start ? 0.f : (a < N ? gpre[a < N ? a : 0] : gradp[g]);
            float inc = sens_increment(Rzv, SX, Rxv, SZ);
            if (edge_node && bgterm) {
              // g lambda (b_{t+2} - b_t), rounded as bnd_sens
              const float* bv = side_col ? bv0 + a : bv0;
              const float du = __fsub_rn(bv[4 * qs], bv[3 * qs]);
              inc = __fadd_rn(inc, __fmul_rn(__fmul_rn(bv[2 * qs], Bs[a * BW + sc]), du));
            }
            gnew = __fadd_rn(gprev, inc);
          }
        }
        float res, vres;
        if constexpr (EDGE) {
          // Stacey mode: one update for every node, w = e1 v + e2 F, with e1 = e2 = 1 off
          // the absorbing edges (selects, so a warp holding an edge column does not diverge)
          const float* bv = side_col ? bv0 + a : bv0;
          const float e1 = edge_node ? bv[0] : 1.f, e2 = edge_node ? bv[qs] : 1.f;
          advance_node_stacey(ADJ, Bs[a * BW + sc], Vs[a * BW + sc], X, Z, ixv, Rxv, izv, Rzv, extra, e1,
                              e2, res, vres);
          if (top_row) {  // free surface
            res = 0.f;
            vres = 0.f;
          }
          if (edge_node && !ADJ && (S.flags & F_ADJ)) S.bnd_hist[(long long)(t + 1) * S.bnd_pitch + bk] = res;
        } else {
          advance_node(ADJ, damp, Bs[a * BW + sc], Vs[a * BW + sc], X, Z, ixv, Rxv, dxv, izv, Rzv,
                       dzv, extra, res, vres);
        }
        out[g] = res;
        vout[g] = vres;
        if (ADJ && grad_on) {
          if (g_fold)
            grad64p[g] = __dadd_rn(g64[a], (double)gnew);
          else
            gradp[g] = gnew;
        }
        bad |= !isfinite(res);
      }
    };
    if (owned) {
      phase_b(std::integral_constant<bool, STC>{});
      zc = rz[N];
      if (ADJ) szc = sz[N];
      if (ADJ && in_win) {  // carry the injection row shared with the next band
        const float carry = sacc[N * NT + tid];
#pragma unroll
        for (int a = 1; a < NP; ++a) sacc[a * NT + tid] = 0.f;
        sacc[tid] = carry;
      }
    }
  }
#if SEM_BND_ASYNC
  if (STC) cp_async_wait_all();  // no edge-value copy outlives the tick
#endif
  if (abort_ez >= 0) {
    // drain the copies still in flight (issued bands from abort_ez on) before leaving
    if (tid == 0) atomicOr(S.status, SEM_ERR_TIMEOUT);
    // issued so far: bands rel < NST, then rel' - 1 + NST at the barrier of each band rel' <
    // the aborting one (final read-out ticks: rel' + NST after each band rel' before it)
    const int ra = abort_ez - ezs;
    const int issued = min(nbands, final_only ? ra + NST : max(NST, ra + NST - 1));
    for (int r = ra; r < issued; ++r) mbar_wait(bars + r % NST, (unsigned)((r / NST) & 1));
    return;
  }
  if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(S.status, SEM_ERR_NONFINITE);
  if constexpr (COH) {
    // the persistent kernel runs the next tick on the same shared memory: every copy has
    // landed and every thread is past its last ring wait, so the barriers are invalidated
    // before the next tick initialises them again (re-initialising a valid mbarrier is
    // undefined)
    __syncthreads();
    if (tid == 0)
      for (int s2 = 0; s2 < NST; ++s2) mbar_inval(bars + s2);
    __syncthreads();
  }
}
#undef Dr
#undef Bt

template <int N>
__global__ void __launch_bounds__(kStripCols, (N <= 4) ? SEM_STRIP_MIN_BLOCKS : 3)
    sem_strip_kernel(const SolveDev* __restrict__ solves, const int* __restrict__ cta_solve,
                     const int* __restrict__ tick_ptr, int unused0, int unused1, int tick_arg) {
  extern __shared__ __align__(128) float smem[];
  __shared__ SolveDev S;
  __shared__ int s_act, s_t, s_seg, s_abort;
  grid_dep_launch();

  const int sid = cta_solve[blockIdx.x];
  {
    const unsigned long long* src = reinterpret_cast<const unsigned long long*>(solves + sid);
    unsigned long long* dst = reinterpret_cast<unsigned long long*>(&S);
    for (int i = threadIdx.x; i < (int)(sizeof(SolveDev) / 8); i += kStripCols) dst[i] = src[i];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int act, t, seg;
    decode(S, (tick_ptr ? *tick_ptr : tick_arg) - S.start_tick, act, t, seg);
    s_act = act; s_t = t; s_seg = seg; s_abort = 0x7fffffff;
  }
  __syncthreads();
  grid_dep_wait();  // the previous tick's fields are complete from here on
  const int act = s_act;
  if (act == A_NONE) return;
  const int t = s_t, seg = s_seg;
  if (act == A_SCALE) {
    if (blockIdx.x == S.tile_base && threadIdx.x == 0) {
      double m = 0.0;
      for (int r = 0; r < S.nrec; ++r) m = fmax(m, S.rmax[r]);
      *S.adj_scale = (m > 0.0 && isfinite(m)) ? ldexp(1.0, -ilogb(m)) : 1.0;
    }
    return;
  }
  if (S.bnd_n > 0) {
    if (act == A_ADJ)
      strip_tick<N, true, false, true>(S, act, t, seg, smem, &s_abort);
    else
      strip_tick<N, false, false, true>(S, act, t, seg, smem, &s_abort);
  } else {
    if (act == A_ADJ)
      strip_tick<N, true, false, false>(S, act, t, seg, smem, &s_abort);
    else
      strip_tick<N, false, false, false>(S, act, t, seg, smem, &s_abort);
  }
}

// ----------------------------------------------------------------------------
// persistent tile kernel: one cooperative launch runs the whole tick program of a
// latency-bound group (small meshes, one solve at a time), with a grid barrier between
// ticks instead of a kernel boundary
// ----------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
// Arrive at and wait on the grid barrier: `count` only grows (target = ticks done x CTAs),
// thread 0 releases the CTA's writes (fence, then the arrival) and polls with acquire
// loads.  Gives up after kWaitNs and returns false (every CTA is resident: cooperative
// launch, so a late CTA is late, not absent).
__device__ __forceinline__ bool grid_barrier(unsigned long long* count, unsigned long long target,
                                             int* s_flag) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(count, 1ull);
    int ok = 1;
    if (ld_acquire_u64(count) < target) {
      const long long t0 = global_ns();
      while (ld_acquire_u64(count) < target)
        if (global_ns() - t0 > kWaitNs) { ok = 0; break; }
    }
    *s_flag = ok;
  }
  __syncthreads();
  return *s_flag != 0;
}

template <int N>
__global__ void __launch_bounds__(256) sem_persist_kernel(const SolveDev* __restrict__ solves,
                                                          const int* __restrict__ cta_solve,
                                                          int tick0, int tick1, int tex, int tez,
                                                          unsigned long long* __restrict__ bar) {
  extern __shared__ float smem[];
  __shared__ SolveDev S;
  __shared__ int s_act, s_t, s_seg, s_ok;
  const int sid = cta_solve[blockIdx.x];
  {
    const unsigned long long* src = reinterpret_cast<const unsigned long long*>(solves + sid);
    unsigned long long* dst = reinterpret_cast<unsigned long long*>(&S);
    for (int i = threadIdx.x; i < (int)(sizeof(SolveDev) / 8); i += blockDim.x) dst[i] = src[i];
  }
  unsigned long long target = 0;
  for (int tick = tick0; tick < tick1; ++tick) {
    __syncthreads();
    if (threadIdx.x == 0) {
      int act, t, seg;
      decode(S, tick - S.start_tick, act, t, seg);
      s_act = act; s_t = t; s_seg = seg;
    }
    __syncthreads();
    const int act = s_act;
#if SEM_TILE_SPLIT
    if (act == A_ADJ)
      tile_tick<N, true, true, true>(S, act, s_t, s_seg, tex, tez, smem);
    else if (act != A_NONE)
      tile_tick<N, true, true, false>(S, act, s_t, s_seg, tex, tez, smem);
#else
    if (act != A_NONE) tile_tick<N, true>(S, act, s_t, s_seg, tex, tez, smem);
#endif
    if (tick + 1 == tick1) break;
    target += gridDim.x;
    if (!grid_barrier(bar, target, &s_ok)) {
      if (threadIdx.x == 0) atomicOr(S.status, SEM_ERR_TIMEOUT);
      return;
    }
  }
}

// ----------------------------------------------------------------------------
// persistent strip kernel: one cooperative launch runs the whole tick program of a group
// of strip chunks that are all resident at once (a single large solve, or a few), so a
// tick costs no launch and no grid drain.  A CTA starts tick t when the eight CTAs around
// it (the only CTAs whose nodes its bands read and use: halo columns, the halo band
// above, the shared row below, and a receiver element's corner node) have published tick
// t - 1; the adjoint-scale tick of a solve takes a
// barrier over that solve's CTAs before and after it.  Every wait is bounded (kWaitNs)
// and ends the launch with SEM_ERR_TIMEOUT.  Bitwise the same arithmetic as the per-tick
// strip kernel (the same strip_tick, with loads of data this launch wrote taken past L1).
// ----------------------------------------------------------------------------
__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u32(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
// Thread i < nn waits until CTA nb[i] has published at least `want` ticks (false after
// kWaitNs); all threads must call it.  Returns true when every wait succeeded.
__device__ __forceinline__ bool wait_neighbours(const unsigned* done, const int* nb, int nn,
                                                unsigned want) {
  bool ok = true;
  if ((int)threadIdx.x < nn) {
    const unsigned* p = done + nb[threadIdx.x];
    if (ld_acquire_u32(p) < want) {
      const long long t0 = global_ns();
      while (ld_acquire_u32(p) < want)
        if (global_ns() - t0 > kWaitNs) { ok = false; break; }
    }
  }
  return __syncthreads_and(ok) != 0;
}

template <int N>
__global__ void __launch_bounds__(kStripCols, (N <= 4) ? SEM_STRIP_MIN_BLOCKS : 3)
    sem_strip_persist_kernel(const SolveDev* __restrict__ solves, const int* __restrict__ cta_solve,
                             int tick0, int tick1, unsigned* __restrict__ done,
                             unsigned long long* __restrict__ sbar) {
  extern __shared__ __align__(128) float smem[];
  __shared__ SolveDev S;
  __shared__ int s_act, s_t, s_seg, s_abort, s_ok;
  __shared__ int s_nb[8], s_nn, s_local;           // neighbour CTAs (kept out of registers)
  __shared__ unsigned long long s_arrivals, s_per_solve;
  const int sid = cta_solve[blockIdx.x];
  {
    const unsigned long long* src = reinterpret_cast<const unsigned long long*>(solves + sid);
    unsigned long long* dst = reinterpret_cast<unsigned long long*>(&S);
    for (int i = threadIdx.x; i < (int)(sizeof(SolveDev) / 8); i += kStripCols) dst[i] = src[i];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int zch = S.zchunk > 0 ? S.zchunk : S.nelz;
    const int nzc = (S.nelz + zch - 1) / zch;
    const int local = blockIdx.x - S.tile_base;
    const int strip = local / nzc, chunk = local - strip * nzc;
    // the eight surrounding CTAs: a receiver element read out of a band can reach the node
    // at a chunk's corner, which the diagonal neighbour owns
    int nn = 0;
    for (int ds = -1; ds <= 1; ++ds)
      for (int dc = -1; dc <= 1; ++dc) {
        const int st = strip + ds, ch = chunk + dc;
        if ((ds || dc) && st >= 0 && st < S.tiles_x && ch >= 0 && ch < nzc)
          s_nb[nn++] = (int)blockIdx.x + ds * nzc + dc;
      }
    s_nn = nn;
    s_local = local;
    s_per_solve = (unsigned long long)S.tiles_x * nzc;
    s_arrivals = 0;  // this solve's barrier target so far
  }
  __syncthreads();
  for (int tick = tick0; tick < tick1; ++tick) {
    if (threadIdx.x == 0) {
      int act, t, seg;
      decode(S, tick - S.start_tick, act, t, seg);
      s_act = act; s_t = t; s_seg = seg; s_abort = 0x7fffffff;
    }
    __syncthreads();
    const int act = s_act;
    bool ok = true;
    if (act == A_SCALE) {
      // every CTA of the solve has read out its receivers; one picks the scale; all see it
      const unsigned long long a1 = s_arrivals + s_per_solve, a2 = a1 + s_per_solve;
      ok = grid_barrier(sbar + sid, a1, &s_ok);
      if (ok && s_local == 0 && threadIdx.x == 0) {
        double m = 0.0;
        for (int r = 0; r < S.nrec; ++r) m = fmax(m, __ldcg(S.rmax + r));
        *S.adj_scale = (m > 0.0 && isfinite(m)) ? ldexp(1.0, -ilogb(m)) : 1.0;
      }
      ok = ok && grid_barrier(sbar + sid, a2, &s_ok);
      if (threadIdx.x == 0) s_arrivals = a2;
    } else if (act != A_NONE) {
      ok = wait_neighbours(done, s_nb, s_nn, (unsigned)(tick - tick0));
      if (ok) {
        // the neighbours' generic-proxy stores come before this tick's bulk / tensor loads
        asm volatile("fence.proxy.async.global;" ::: "memory");
        if (S.bnd_n > 0) {
          if (act == A_ADJ)
            strip_tick<N, true, true, true>(S, act, s_t, s_seg, smem, &s_abort);
          else
            strip_tick<N, false, true, true>(S, act, s_t, s_seg, smem, &s_abort);
        } else {
          if (act == A_ADJ)
            strip_tick<N, true, true, false>(S, act, s_t, s_seg, smem, &s_abort);
          else
            strip_tick<N, false, true, false>(S, act, s_t, s_seg, smem, &s_abort);
        }
        __syncthreads();
        if (s_abort != 0x7fffffff) return;  // a copy wait gave up: status set, copies drained
      }
    }
    if (!ok) {
      if (threadIdx.x == 0) atomicOr(S.status, SEM_ERR_TIMEOUT);
      return;
    }
    __syncthreads();  // every thread's stores of this tick are issued
    if (threadIdx.x == 0) {
      __threadfence();
      st_release_u32(done + blockIdx.x, (unsigned)(tick - tick0 + 1));
    }
  }
}

// Diagnostics of the device waits' time limits, without any fault: which = 0 waits on an
// mbarrier whose expected bytes never arrive (no copy is issued), 1 on a grid barrier one
// arrival short of its target (cooperative launch of 2 CTAs), 2 on a grid barrier that
// completes.  A wait that gives up sets SEM_ERR_TIMEOUT in *status.
__global__ void wait_probe_kernel(int which, unsigned long long* bar, int* status) {
  __shared__ unsigned long long mb;
  __shared__ int s_ok;
  if (which == 0) {
    if (threadIdx.x == 0) {
      mbar_init(&mb, 1);
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
      mbar_expect_tx(&mb, 16u);  // the only arrival, and 16 bytes that never come
    }
    __syncthreads();
    if (!mbar_wait(&mb, 0) && threadIdx.x == 0) atomicOr(status, SEM_ERR_TIMEOUT);
    return;
  }
  const unsigned long long target = gridDim.x + (which == 1 ? 1ull : 0ull);
  if (!grid_barrier(bar, target, &s_ok) && threadIdx.x == 0) atomicOr(status, SEM_ERR_TIMEOUT);
}

__global__ void tick_advance_kernel(int* tick) { *tick += 1; }

// c (float64, reference order) -> c^2 (float32, pitched grid)
__global__ void set_c2_kernel(const double* __restrict__ c, const int* __restrict__ pos,
                              float* __restrict__ c2, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double v = c[i];
    c2[pos[i]] = (float)(v * v);
  }
}

__global__ void copy_status_kernel(const int* __restrict__ st, int* __restrict__ out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *out = *st;
}

// Per-solve inputs and outputs of one sem_run group, for the batched set-up and output
// kernels (one grid row per solve).
struct SolveIo {
  const double* vel;      // [npoints] velocity, reference node order
  const int* pos;         // [npoints] grid offset of each node
  float* c2;              // c^2 field
  int npoints, nzero;
  char* zp[8];            // workspace ranges that must start at zero (256-byte aligned,
  long long zb[8];        //   lengths multiples of 16 bytes)
  double* grad_out;       // or null
  const double* gacc;     // dJ/dc^2 accumulator (float64, scaled)
  const double* adj_scale;
  double inv_sigma2;
  const double* misfit;   // [nrec]
  int nrec;
  double* loglik_out;     // or null
  const int* st;          // workspace status word
  int* status_out;        // or null
  // Stacey mode: per boundary slot the node's reference index and the plan's alpha and
  // gamma; the set-up writes e1, e2 and g of this solve's velocity into bnd_coef
  int bnd_n, bnd_pitch;
  const int* bnd_ref;
  const double* bnd_alpha;
  const double* bnd_gamma;
  float* bnd_coef;
};

// clears every solve's zero-start state and stages c^2 (row blockIdx.y = solve)
__global__ void batch_setup_kernel(const SolveIo* __restrict__ io, int s0) {
  const SolveIo& s = io[s0 + blockIdx.y];
  const long long t0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (int r = 0; r < s.nzero; ++r) {
    uint4* p = reinterpret_cast<uint4*>(s.zp[r]);
    const long long n16 = s.zb[r] >> 4;
    for (long long i = t0; i < n16; i += stride) p[i] = make_uint4(0u, 0u, 0u, 0u);
  }
  for (long long i = t0; i < s.npoints; i += stride) {
    const double v = s.vel[i];
    s.c2[s.pos[i]] = (float)(v * v);
  }
  // Stacey mode: a = c alpha, e1 = (1 - a) / (1 + a), e2 = 1 / (1 + a), g = gamma / c
  for (long long k = t0; k < s.bnd_n; k += stride) {
    const int ref = s.bnd_ref[k];
    float e1 = 0.f, e2 = 0.f, g = 0.f;
    if (ref >= 0) {
      const double c = s.vel[ref];
      const double a = c * s.bnd_alpha[k];
      e1 = (float)((1.0 - a) / (1.0 + a));
      e2 = (float)(1.0 / (1.0 + a));
      g = (float)(s.bnd_gamma[k] / c);
    }
    s.bnd_coef[k] = e1;
    s.bnd_coef[s.bnd_pitch + k] = e2;
    s.bnd_coef[2LL * s.bnd_pitch + k] = g;
  }
}

// gradient in reference node order, log-likelihood and status of every solve:
//   grad_out[i] = 2 c_i * acc[pos_i] * inv_sigma2 / adj_scale   (dJ/dc = 2c dJ/dc^2,
//     core.py:84; adj_scale is a power of two, so the division is exact)
//   loglik = -0.5 inv_sigma2 sum_r misfit_r   (fixed receiver order: deterministic)
__global__ void batch_output_kernel(const SolveIo* __restrict__ io, int s0) {
  const SolveIo& s = io[s0 + blockIdx.y];
  if (s.grad_out) {
    const double scale = s.inv_sigma2 / *s.adj_scale;  // exact: adj_scale is a power of two
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < s.npoints;
         i += (long long)gridDim.x * blockDim.x)
      s.grad_out[i] = 2.0 * s.vel[i] * s.gacc[s.pos[i]] * scale;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (s.loglik_out) {
      double m = 0.0;
      for (int r = 0; r < s.nrec; ++r) m += s.misfit[r];
      *s.loglik_out = -0.5 * m * s.inv_sigma2;
    }
    if (s.status_out) *s.status_out = *s.st;
  }
}

// ----------------------------------------------------------------------------
// Scratch of the allocation-free forward entry point (sem_forward_noalloc).  Every
// GPU that loads this library holds it until the process exits.  Host code must not
// use the symbol's name as an address: it takes the device address once per device
// with cudaGetSymbolAddress.
// ----------------------------------------------------------------------------
constexpr size_t kNoAllocScratchBytes = 32u << 20;  // 32 MiB
constexpr int kNoAllocTile = 8;                      // 8x8-element tiles, 256 threads
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// writes the solve descriptor (passed by value), the CTA map and the tick counter
// into the scratch, and clears the state that must start at zero
__global__ void noalloc_setup_kernel(SolveDev d, SolveDev* desc, int* cta, int ncta, int* tick,
                                     float* zero_f, long long nzero_f, int* status) {
  const long long i0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  if (i0 == 0) { *desc = d; *tick = 0; *status = 0; }
  for (long long i = i0; i < ncta; i += stride) cta[i] = 0;
  for (long long i = i0; i < nzero_f; i += stride) zero_f[i] = 0.f;
}

}  // namespace

// ============================================================================
// host side
// ============================================================================
struct sem_plan_s {
  int nelx, nelz, npol, nt, npoints, nxg, nzg, pitch, nrec, src_gx, src_gz, device;
  double dt;
  long long fstride;
  char* noalloc_scratch = nullptr;  // device address of the allocation-free entry point's
                                    // scratch array on this plan's device
  int bnd_n = 0;                    // Stacey mode: boundary slots (0: the sponge)
  int* bnd_ref = nullptr;
  double* bnd_alpha = nullptr;
  double* bnd_gamma = nullptr;
  float* D = nullptr;
  float* beta = nullptr;
  float* tx = nullptr;
  float* tz = nullptr;
  float* src_term = nullptr;
  int* rec_base = nullptr;
  float* rec_w = nullptr;
  int* node_pos = nullptr;
  std::vector<int> h_rec_base;
  // receiver lists per tile (tile kernel, key (tile_ex, tile_ez)) or per strip band
  // (strip kernel, key (-1, elements per strip)): device arrays rec_off/ids, inj_off/ids
  struct Lists { int* rec_off; int* rec_ids; int* inj_off; int* inj_ids; };
  mutable std::map<std::pair<int, int>, Lists> lists;
  mutable std::mutex mu;
};

namespace {

template <class T>
int upload(T** dst, const T* src, size_t n) {
  CUDA_TRY(cudaMalloc((void**)dst, std::max<size_t>(n, 1) * sizeof(T)));
  if (n) CUDA_TRY(cudaMemcpy(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice));
  return SEM_OK;
}

// fills c_D[N] / c_B[N] on the current device once; later plans of the same order must
// bring the same operators
int set_order_constants(int dev, int N, const double* D, const double* beta) {
  static std::mutex mu;
  static std::map<std::pair<int, int>, std::vector<float>> have;
  const int NP = N + 1;
  std::vector<float> v((size_t)NP * NP + NP);
  for (int i = 0; i < NP * NP; ++i) v[i] = (float)D[i];
  for (int i = 0; i < NP; ++i) v[NP * NP + i] = (float)beta[i];
  std::lock_guard<std::mutex> lk(mu);
  auto it = have.find(std::make_pair(dev, N));
  if (it != have.end()) {
    if (it->second != v)
      return fail(SEM_ERR_ARG, "GLL operators differ from an earlier plan of the same order");
    return SEM_OK;
  }
  CUDA_TRY(cudaMemcpyToSymbol(c_D, v.data(), sizeof(float) * NP * NP, sizeof(float) * 64 * N));
  CUDA_TRY(cudaMemcpyToSymbol(c_B, v.data() + NP * NP, sizeof(float) * NP, sizeof(float) * 8 * N));
  std::vector<float2> v2(v.size());
  for (size_t i = 0; i < v.size(); ++i) v2[i] = make_float2(v[i], v[i]);
  CUDA_TRY(cudaMemcpyToSymbol(c_D2, v2.data(), sizeof(float2) * NP * NP, sizeof(float2) * 64 * N));
  CUDA_TRY(cudaMemcpyToSymbol(c_B2, v2.data() + NP * NP, sizeof(float2) * NP, sizeof(float2) * 8 * N));
  have[std::make_pair(dev, N)] = v;
  return SEM_OK;
}

// The dynamic shared-memory limit is an attribute of the kernel function, shared by every
// host thread that launches it.  It is only ever raised here, so a launch on one thread
// never finds the limit lowered below its own size by a launch of another thread (the
// strip and tile kernels of one order run with different sizes for forward-only and
// adjoint groups).
cudaError_t raise_smem_limit(const void* fn, size_t smem) {
  static std::mutex mu;
  static std::map<std::pair<int, const void*>, size_t> cur;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(mu);
  size_t& c = cur[std::make_pair(dev, fn)];
  if (smem <= c) return cudaSuccess;
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) c = smem;
  return e;
}

int upload_f32(float** dst, const double* src, size_t n) {
  std::vector<float> tmp(n);
  for (size_t i = 0; i < n; ++i) tmp[i] = (float)src[i];
  return upload(dst, tmp.data(), n);
}

long long round_up(long long v, long long m) { return (v + m - 1) / m * m; }

int tiles_of(const sem_plan_s* p, int tex, int tez, int* tx, int* tz) {
  *tx = (p->nelx + tex - 1) / tex;
  *tz = (p->nelz + tez - 1) / tez;
  return (*tx) * (*tz);
}

// strip kernel: strips of a plan and elements per strip (balanced)
int strips_of(const sem_plan_s* p, int* ew_out) {
  const int ewm = strip_ew_max(p->npol);
  int ns = (p->nelx + ewm - 1) / ewm;
  const int ew = (p->nelx + ns - 1) / ns;
  ns = (p->nelx + ew - 1) / ew;
  if (ew_out) *ew_out = ew;
  return ns;
}
constexpr int kMinChunk = 4;  // element rows per strip CTA at least: halo band <= 1/4 extra
// element rows per strip CTA: full height when the strips alone give every SM two CTAs,
// else chunks of at least kMinChunk rows so that strips x chunks comes near four per SM
int strip_zchunk(long long total_strips, int nelz_max, int sms, int forced) {
  if (forced > 0) return forced;
  if (total_strips >= 2LL * sms) return nelz_max;
  const long long want = (4LL * sms + total_strips - 1) / total_strips;  // chunks per strip
  return std::max(kMinChunk, (int)((nelz_max + want - 1) / want));
}
// automatic variant choice: strips when the chunked strip grid gives every SM two CTAs
bool strip_fills(long long min_chunk_ctas, int sms) { return min_chunk_ctas >= 2LL * sms; }
// automatic tile shape of the tile kernel: the finest tiling of the batch whose CTAs all
// fit on the GPU at once (one wave, counted with the tile kernel's occupancy at each
// candidate's shared memory), else 8x8.  A tick of a small batch is latency-bound: smaller
// tiles finish sooner while they stay resident, but a second wave doubles the tick (100x50
// elements at N = 4, 3 CTAs per SM: 4x3 tiles, 425 CTAs, run 9 % faster than 4x4 tiles,
// 325 CTAs, and 3x3 tiles, 578 CTAs, take 40 % longer).
typedef void (*KernelFn)(const SolveDev*, const int*, const int*, int, int, int);
KernelFn kernel_for(int N);
void auto_tile(const sem_solve_t* sv, int n, int sms, int threads, int* tex, int* tez) {
  static const int cand[][2] = {{8, 8}, {8, 4}, {4, 4}, {4, 3}, {4, 2}, {2, 4}, {2, 2}, {2, 1}};
  const int nc = (int)(sizeof(cand) / sizeof(cand[0]));
  bool adj = false;
  for (int i = 0; i < n; ++i) adj |= (sv[i].flags & SEM_F_ADJOINT) != 0;
  int best = 0;
  long long best_tiles = -1;
  for (int c = 0; c < nc; ++c) {
    // per order: tiles over the batch and CTAs resident per SM
    long long tiles[kMaxN + 1] = {};
    for (int i = 0; i < n; ++i) {
      int tx, tz;
      tiles[sv[i].plan->npol] += tiles_of(sv[i].plan, cand[c][0], cand[c][1], &tx, &tz);
    }
    double load = 0.0;
    long long total = 0;
    for (int N = 1; N <= kMaxN; ++N) {
      if (!tiles[N]) continue;
      const size_t smem = (size_t)smem_floats(N, cand[c][0], cand[c][1], adj) * sizeof(float);
      KernelFn fn = kernel_for(N);
      int nb = 0;
      if (smem > 227 * 1024 || raise_smem_limit((const void*)fn, smem) != cudaSuccess ||
          cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, threads, smem) != cudaSuccess || nb < 1) {
        load = 2.0;
        break;
      }
      load += (double)tiles[N] / ((double)nb * sms);
      total += tiles[N];
    }
    if (load <= 1.0 && total > best_tiles) {
      best = c;
      best_tiles = total;
    }
  }
  *tex = cand[best][0];
  *tez = cand[best][1];
}

int upload_lists(const sem_plan_s* p, std::pair<int, int> key, std::vector<std::vector<int>>& rec,
                 std::vector<std::vector<int>>& inj, sem_plan_s::Lists* out) {
  const int nl = (int)rec.size();
  for (auto& v : inj)
    if ((int)v.size() > kMaxInj) return fail(SEM_ERR_ARG, "too many receivers in one tile; use smaller tiles");
  auto flat = [&](std::vector<std::vector<int>>& v, std::vector<int>& off, std::vector<int>& ids) {
    off.assign(nl + 1, 0);
    for (int i = 0; i < nl; ++i) off[i + 1] = off[i] + (int)v[i].size();
    for (auto& x : v) ids.insert(ids.end(), x.begin(), x.end());
  };
  std::vector<int> ro, ri, io, ii;
  flat(rec, ro, ri);
  flat(inj, io, ii);
  sem_plan_s::Lists L{};
  int rc;
  if ((rc = upload(&L.rec_off, ro.data(), ro.size()))) return rc;
  if ((rc = upload(&L.rec_ids, ri.data(), ri.size()))) return rc;
  if ((rc = upload(&L.inj_off, io.data(), io.size()))) return rc;
  if ((rc = upload(&L.inj_ids, ii.data(), ii.size()))) return rc;
  p->lists[key] = L;
  *out = L;
  return SEM_OK;
}

int get_lists(const sem_plan_s* p, int tex, int tez, sem_plan_s::Lists* out) {
  std::lock_guard<std::mutex> lk(p->mu);
  auto key = std::make_pair(tex, tez);
  auto it = p->lists.find(key);
  if (it != p->lists.end()) { *out = it->second; return SEM_OK; }
  int ntx, ntz;
  const int ntiles = tiles_of(p, tex, tez, &ntx, &ntz);
  const int N = p->npol;
  std::vector<std::vector<int>> rec(ntiles), inj(ntiles);
  for (int r = 0; r < p->nrec; ++r) {
    const int bx = p->h_rec_base[2 * r], bz = p->h_rec_base[2 * r + 1];
    const int ex = bx / N, ez = bz / N;
    rec[(ez / tez) * ntx + (ex / tex)].push_back(r);
    std::vector<int> seen;
    for (int j = 0; j <= N; ++j)
      for (int i = 0; i <= N; ++i) {
        const int ox = std::min((bx + i) / (tex * N), ntx - 1);
        const int oz = std::min((bz + j) / (tez * N), ntz - 1);
        const int tt = oz * ntx + ox;
        if (std::find(seen.begin(), seen.end(), tt) == seen.end()) seen.push_back(tt);
      }
    for (int tt : seen) inj[tt].push_back(r);
  }
  return upload_lists(p, key, rec, inj, out);
}

// strip kernel lists, indexed strip * nelz + element row
int get_strip_lists(const sem_plan_s* p, int ew, sem_plan_s::Lists* out) {
  std::lock_guard<std::mutex> lk(p->mu);
  auto key = std::make_pair(-1, ew);
  auto it = p->lists.find(key);
  if (it != p->lists.end()) { *out = it->second; return SEM_OK; }
  const int N = p->npol;
  const int ns = (p->nelx + ew - 1) / ew;
  std::vector<std::vector<int>> rec((size_t)ns * p->nelz), inj((size_t)ns * p->nelz);
  for (int r = 0; r < p->nrec; ++r) {
    const int bx = p->h_rec_base[2 * r], bz = p->h_rec_base[2 * r + 1];
    const int ex = bx / N, ez = bz / N;
    rec[(size_t)(ex / ew) * p->nelz + ez].push_back(r);
    for (int s = 0; s < ns; ++s) {
      const int sx0 = s * ew * N;
      const int so1 = (std::min((s + 1) * ew, p->nelx) == p->nelx) ? p->nxg : (s + 1) * ew * N;
      if (bx + N >= sx0 && bx < so1) inj[(size_t)s * p->nelz + ez].push_back(r);
    }
  }
  for (auto& v : inj)
    if ((int)v.size() > kStripInj) return fail(SEM_ERR_ARG, "too many receivers in one strip band");
  return upload_lists(p, key, rec, inj, out);
}

KernelFn strip_kernel_for(int N) {
  switch (N) {
    case 1: return sem_strip_kernel<1>;
    case 2: return sem_strip_kernel<2>;
    case 3: return sem_strip_kernel<3>;
    case 4: return sem_strip_kernel<4>;
    case 5: return sem_strip_kernel<5>;
    case 6: return sem_strip_kernel<6>;
    case 7: return sem_strip_kernel<7>;
  }
  return nullptr;
}

KernelFn kernel_for(int N) {
  switch (N) {
    case 1: return sem_tick_kernel<1>;
    case 2: return sem_tick_kernel<2>;
    case 3: return sem_tick_kernel<3>;
    case 4: return sem_tick_kernel<4>;
    case 5: return sem_tick_kernel<5>;
    case 6: return sem_tick_kernel<6>;
    case 7: return sem_tick_kernel<7>;
  }
  return nullptr;
}

typedef void (*StripPersistFn)(const SolveDev*, const int*, int, int, unsigned*, unsigned long long*);
StripPersistFn strip_persist_kernel_for(int N) {
  switch (N) {
    case 1: return sem_strip_persist_kernel<1>;
    case 2: return sem_strip_persist_kernel<2>;
    case 3: return sem_strip_persist_kernel<3>;
    case 4: return sem_strip_persist_kernel<4>;
    case 5: return sem_strip_persist_kernel<5>;
    case 6: return sem_strip_persist_kernel<6>;
    case 7: return sem_strip_persist_kernel<7>;
  }
  return nullptr;
}

typedef void (*PersistFn)(const SolveDev*, const int*, int, int, int, int, unsigned long long*);
PersistFn persist_kernel_for(int N) {
  switch (N) {
    case 1: return sem_persist_kernel<1>;
    case 2: return sem_persist_kernel<2>;
    case 3: return sem_persist_kernel<3>;
    case 4: return sem_persist_kernel<4>;
    case 5: return sem_persist_kernel<5>;
    case 6: return sem_persist_kernel<6>;
    case 7: return sem_persist_kernel<7>;
  }
  return nullptr;
}

struct Workspace {
  long long c2, W, V, ckpt, ring, L, Mu, grad, grad64, misfit, status;  // byte offsets
  long long bnd_coef, bnd_hist;  // Stacey mode (-1 when absent)
  long long bytes;
};
// floats per row of the boundary tables
inline int bnd_pitch_of(const sem_plan_s* p) { return (p->bnd_n + 63) / 64 * 64; }

// The strip kernel's band loads: one tiled tensor map per solve over its workspace seen as
// [field slot][row][column] floats (c2, W, V, checkpoints, ring, L and Mu all start at
// multiples of the field stride), box = strip_bw columns x N+1 rows of one field.
typedef CUresult (*TensorMapEncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                           const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                           const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                           CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
TensorMapEncodeTiledFn tensor_map_encoder() {
  static TensorMapEncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<TensorMapEncodeTiledFn>(f);
    cudaGetLastError();
  });
  return fn;
}
int encode_band_map(CUtensorMap* m, char* ws_base, const sem_plan_s* p, long long nslots) {
  TensorMapEncodeTiledFn enc = tensor_map_encoder();
  if (!enc) return fail(SEM_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
  const cuuint64_t dims[3] = {(cuuint64_t)p->pitch, (cuuint64_t)p->nzg, (cuuint64_t)nslots};
  const cuuint64_t strides[2] = {(cuuint64_t)p->pitch * 4, (cuuint64_t)p->fstride * 4};
  const cuuint32_t box[3] = {(cuuint32_t)strip_bw(p->npol), (cuuint32_t)(p->npol + 1), 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, ws_base, dims, strides, box, estr,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? SEM_OK : fail(SEM_ERR_CUDA, "tensor map encoding failed");
}
// float-field slots of a workspace (everything before the gradient / the misfit)
long long field_slots(const Workspace& w, const sem_plan_s* p, bool adj) {
  return (adj ? w.grad : w.misfit) / (p->fstride * 4);
}

Workspace layout(const sem_plan_s* p, int flags, int k, int* nseg_out) {
  Workspace w{};
  const long long F = p->fstride * 4;  // bytes per float field (multiple of 256)
  const bool adj = flags & SEM_F_ADJOINT;
  const int nseg = adj ? (p->nt + k - 1) / k : 1;
  long long o = 0;
  w.c2 = o; o += F;
  w.W = o; o += 2 * F;
  w.V = o; o += F;
  if (adj) {
    w.ckpt = o; o += (long long)2 * nseg * F;
    w.ring = o; o += (long long)(k + 1) * F;
    w.L = o; o += 2 * F;
    w.Mu = o; o += F;
    w.grad = o; o += F;
    w.grad64 = o; o += 2 * F;  // float64 field
  }
  w.misfit = o; o += round_up((long long)(2 * p->nrec + 1) * 8, 256);  // misfit, rmax, scale
  w.status = o; o += 256;
  w.bnd_coef = w.bnd_hist = -1;
  if (p->bnd_n > 0) {
    const long long row = (long long)bnd_pitch_of(p) * 4;  // bytes, a multiple of 256
    w.bnd_coef = o; o += 3 * row;                          // e1, e2, g
    if (adj) { w.bnd_hist = o; o += (long long)(p->nt + 1) * row; }  // b_t of the slots
  }
  w.bytes = o;
  *nseg_out = nseg;
  return w;
}

}  // namespace

struct sem_batch_s {
  int device = -1;
  char* arena = nullptr;
  long long arena_bytes = 0;
  int* d_tick = nullptr;
  SolveDev* d_solves = nullptr;
  int solves_cap = 0;
  int* d_cta = nullptr;
  long long cta_cap = 0;
  long long last_launches = 0;
  int last_kernel = 0;
  int last_zchunk = 0;
  int last_tile_ex = 0, last_tile_ez = 0;
  int last_groups = 0;
  long long last_ticks = 0;             // tick rounds of the last sem_run (all groups)
  std::vector<cudaEvent_t> tick_ev;     // per group: before / after its tick loop
  SolveIo* d_io = nullptr;              // per-solve set-up / output table of a group
  int io_cap = 0;
  std::vector<SolveIo> h_io;
  int tick_ev_used = 0;
  std::vector<SolveDev> h_solves;
  std::vector<int> h_cta;
  CUtensorMap* d_tmaps = nullptr;       // strip kernel: band-load tensor map of each solve
  int tmaps_cap = 0;
  std::vector<CUtensorMap> h_tmaps;
  char* d_sync = nullptr;               // persistent strip kernel: per-CTA tick counters and
  long long sync_cap = 0;               //   per-solve barrier counters
};

extern "C" {

const char* sem_last_error(void) { return g_err.c_str(); }

int sem_plan_create(const sem_plan_desc_t* d, sem_plan_t** out) {
  if (!d || !out) return fail(SEM_ERR_ARG, "null argument");
  if (d->npol < 1 || d->npol > kMaxN) return fail(SEM_ERR_UNSUPPORTED, "polynomial order must be 1..7");
  if (d->nelx < 1 || d->nelz < 1 || d->nt < 1 || d->nrec < 0)
    return fail(SEM_ERR_ARG, "bad mesh / nt / nrec");
  const int nxg = d->nelx * d->npol + 1, nzg = d->nelz * d->npol + 1;
  if ((long long)nxg * nzg != d->npoints) return fail(SEM_ERR_ARG, "npoints != nxg*nzg");
  // node offsets within a field are 32-bit in the kernels
  if ((long long)round_up(nxg, 32) * nzg >= (1LL << 31) - 64)
    return fail(SEM_ERR_UNSUPPORTED, "mesh too large: a field must hold fewer than 2^31 nodes");
  if (d->src_gx < 0 || d->src_gx >= nxg || d->src_gz < 0 || d->src_gz >= nzg)
    return fail(SEM_ERR_ARG, "source node outside the mesh");
  auto* p = new sem_plan_s();
  p->nelx = d->nelx; p->nelz = d->nelz; p->npol = d->npol; p->nt = d->nt;
  p->npoints = d->npoints; p->nxg = nxg; p->nzg = nzg; p->nrec = d->nrec;
  p->src_gx = d->src_gx; p->src_gz = d->src_gz; p->dt = d->dt;
  p->pitch = (int)round_up(nxg, 32);
  p->fstride = round_up((long long)p->pitch * nzg, 64);
  cudaGetDevice(&p->device);
  const int NP = d->npol + 1;
  int rc = SEM_OK;
  std::vector<int> pos(d->npoints);
  for (int i = 0; i < d->npoints; ++i) {
    const long long g = d->node_grid[i];
    if (g < 0 || g >= d->npoints) { delete p; return fail(SEM_ERR_ARG, "node_grid out of range"); }
    pos[i] = (int)((g / nxg) * p->pitch + (g % nxg));
  }
  p->h_rec_base.assign(d->rec_base, d->rec_base + 2 * d->nrec);
  for (int r = 0; r < d->nrec; ++r) {
    const int bx = p->h_rec_base[2 * r], bz = p->h_rec_base[2 * r + 1];
    if (bx < 0 || bz < 0 || bx % d->npol || bz % d->npol || bx + d->npol > nxg - 1 ||
        bz + d->npol > nzg - 1) {
      delete p;
      return fail(SEM_ERR_ARG, "receiver element base outside the mesh");
    }
  }
  if ((rc = set_order_constants(p->device, d->npol, d->gll_D, d->gll_beta)) ||
      (rc = upload_f32(&p->D, d->gll_D, NP * NP)) || (rc = upload_f32(&p->beta, d->gll_beta, NP)) ||
      (rc = upload_f32(&p->tx, d->tab_x, 3 * nxg)) || (rc = upload_f32(&p->tz, d->tab_z, 3 * nzg)) ||
      (rc = upload_f32(&p->src_term, d->src_term, d->nt)) ||
      (rc = upload(&p->rec_base, d->rec_base, 2 * (size_t)d->nrec)) ||
      (rc = upload_f32(&p->rec_w, d->rec_w, (size_t)d->nrec * NP * NP)) ||
      (rc = upload(&p->node_pos, pos.data(), pos.size()))) {
    sem_plan_destroy(p);
    return rc;
  }
  if (d->boundary_mode == 1) {
    if (d->bnd_n != 2 * nzg + nxg || !d->bnd_ref || !d->bnd_alpha || !d->bnd_gamma) {
      sem_plan_destroy(p);
      return fail(SEM_ERR_ARG, "Stacey mode needs bnd_n = 2 nzg + nxg and the three boundary tables");
    }
    for (int k = 0; k < d->bnd_n; ++k)
      if (d->bnd_ref[k] >= d->npoints) {
        sem_plan_destroy(p);
        return fail(SEM_ERR_ARG, "bnd_ref out of range");
      }
    p->bnd_n = d->bnd_n;
    if ((rc = upload(&p->bnd_ref, d->bnd_ref, d->bnd_n)) || (rc = upload(&p->bnd_alpha, d->bnd_alpha, d->bnd_n)) ||
        (rc = upload(&p->bnd_gamma, d->bnd_gamma, d->bnd_n))) {
      sem_plan_destroy(p);
      return rc;
    }
  } else if (d->boundary_mode != 0) {
    sem_plan_destroy(p);
    return fail(SEM_ERR_ARG, "boundary_mode must be 0 (sponge) or 1 (Stacey sides and bottom, free top)");
  }
  {
    sem_plan_s::Lists L;  // lists of the default 8x8 tiles, used by sem_forward_noalloc
    if ((rc = get_lists(p, kNoAllocTile, kNoAllocTile, &L))) {
      sem_plan_destroy(p);
      return rc;
    }
  }
  {
    // device address of sem_forward_noalloc's scratch array, taken here (set-up, this
    // plan's device current) so that the entry point itself loads nothing and looks up
    // nothing; the array's host-side name is not a device address
    void* ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess) {
      sem_plan_destroy(p);
      return fail(SEM_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
    }
    p->noalloc_scratch = (char*)ptr;
  }
  *out = p;
  return SEM_OK;
}

int sem_plan_destroy(sem_plan_t* p) {
  if (!p) return SEM_OK;
  cudaFree(p->D); cudaFree(p->beta); cudaFree(p->tx); cudaFree(p->tz); cudaFree(p->src_term);
  cudaFree(p->rec_base); cudaFree(p->rec_w); cudaFree(p->node_pos);
  cudaFree(p->bnd_ref); cudaFree(p->bnd_alpha); cudaFree(p->bnd_gamma);
  for (auto& kv : p->lists) {
    cudaFree(kv.second.rec_off); cudaFree(kv.second.rec_ids);
    cudaFree(kv.second.inj_off); cudaFree(kv.second.inj_ids);
  }
  delete p;
  return SEM_OK;
}

int64_t sem_plan_workspace_bytes(const sem_plan_t* p, int32_t flags, int32_t k) {
  int nseg;
  return layout(p, flags, std::max(2, (int)k), &nseg).bytes;
}

int sem_batch_create(sem_batch_t** out) {
  if (!out) return fail(SEM_ERR_ARG, "null argument");
  auto* b = new sem_batch_s();
  cudaGetDevice(&b->device);
  if (cudaMalloc((void**)&b->d_tick, 256) != cudaSuccess) {
    delete b;
    return fail(SEM_ERR_OOM, "cudaMalloc tick");
  }
  *out = b;
  return SEM_OK;
}

int sem_batch_destroy(sem_batch_t* b) {
  if (!b) return SEM_OK;
  for (cudaEvent_t e : b->tick_ev) cudaEventDestroy(e);
  cudaFree(b->d_io);
  cudaFree(b->arena); cudaFree(b->d_tick); cudaFree(b->d_solves); cudaFree(b->d_cta); cudaFree(b->d_tmaps);
  cudaFree(b->d_sync);
  delete b;
  return SEM_OK;
}

int64_t sem_batch_last_launches(const sem_batch_t* b) { return b ? b->last_launches : -1; }

int32_t sem_batch_last_kernel(const sem_batch_t* b) { return b ? b->last_kernel : -1; }

}  // extern "C"

// One group of solves run to completion: the whole batch, or one group of an automatic
// schedule (solves then carry the group's checkpoint interval).
static int run_group(sem_batch_t* b, const sem_solve_t* solves, int32_t n,
                     const sem_launch_cfg_t& cfg, cudaStream_t stream) {
  if (n == 0) return SEM_OK;

  // ---- validate and lay out workspaces
  std::vector<Workspace> ws(n);
  std::vector<int> nseg(n), kk(n), prog(n);
  long long total = 0;
  for (int i = 0; i < n; ++i) {
    const sem_solve_t& s = solves[i];
    if (!s.plan || !s.velocity || !s.rec_out) return fail(SEM_ERR_ARG, "solve missing plan/velocity/rec_out");
    const bool adj = s.flags & SEM_F_ADJOINT;
    if (adj && !(s.flags & SEM_F_SHIFT)) return fail(SEM_ERR_ARG, "adjoint requires the shifted receiver convention");
    if ((adj || (s.flags & SEM_F_MISFIT)) && !s.y_obs) return fail(SEM_ERR_ARG, "y_obs required");
    if (s.decim < 1 || s.it0 < 0 || s.it1 > s.plan->nt || s.it0 >= s.it1)
      return fail(SEM_ERR_ARG, "bad misfit window");
    kk[i] = adj ? std::max(2, std::min((int)s.ckpt_k, s.plan->nt)) : 2;
    ws[i] = layout(s.plan, s.flags, kk[i], &nseg[i]);
    total += ws[i].bytes;
    const int nt = s.plan->nt;
    prog[i] = nt + ((s.flags & SEM_F_SHIFT) ? 1 : 0) + (adj ? 1 + nt + kk[i] * (nseg[i] - 1) : 0);
  }
  // kernel variant: strips (chunked in z when the strips alone do not fill the GPU) when
  // that grid gives every SM two CTAs, tiles otherwise
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  long long total_strips = 0, min_chunk_ctas = 0;
  int nelz_max = 1;
  for (int i = 0; i < n; ++i) {
    const sem_plan_s* p = solves[i].plan;
    const int ns = strips_of(p, nullptr);
    total_strips += ns;
    min_chunk_ctas += (long long)ns * ((p->nelz + kMinChunk - 1) / kMinChunk);
    nelz_max = std::max(nelz_max, p->nelz);
  }
  bool use_strip = (cfg.kernel == 2 || cfg.kernel == 4);
  if (cfg.kernel == 0) use_strip = strip_fills(min_chunk_ctas, sms);
  const int zchunk = use_strip ? strip_zchunk(total_strips, nelz_max, sms, cfg.strip_bands) : 0;
  b->last_kernel = use_strip ? 2 : 1;
  b->last_zchunk = zchunk;
  if (total > b->arena_bytes) {
    cudaFree(b->arena);
    b->arena = nullptr;
    b->arena_bytes = 0;
    CUDA_TRY(cudaMalloc((void**)&b->arena, total));
    b->arena_bytes = total;
  }

  // ---- group by polynomial order, build descriptors and CTA maps
  std::vector<int> order(n);
  for (int i = 0; i < n; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(),
                   [&](int x, int y) { return solves[x].plan->npol < solves[y].plan->npol; });
  b->h_solves.assign(n, SolveDev{});
  if (use_strip && n > b->tmaps_cap) {
    cudaFree(b->d_tmaps);
    b->d_tmaps = nullptr;
    b->tmaps_cap = 0;
    CUDA_TRY(cudaMalloc((void**)&b->d_tmaps, sizeof(CUtensorMap) * n));
    b->tmaps_cap = n;
  }
  if (use_strip) b->h_tmaps.resize(n);
  b->h_cta.clear();
  struct Group { int N; long long cta0, ncta; bool adj, stc; };
  std::vector<Group> groups;
  long long off = 0;
  int max_prog = 0;
  std::vector<long long> base(n);
  for (int oi = 0; oi < n; ++oi) {
    const int i = order[oi];
    const sem_solve_t& s = solves[i];
    const sem_plan_s* p = s.plan;
    if (p->device != b->device) return fail(SEM_ERR_ARG, "plan and batch on different devices");
    sem_plan_s::Lists L;
    int ntx, ntz, ntiles, rc;
    if (use_strip) {
      ntx = strips_of(p, &ntz);                    // strips, elements per strip
      ntiles = ntx * ((p->nelz + zchunk - 1) / zchunk);
      rc = get_strip_lists(p, ntz, &L);
    } else {
      ntiles = tiles_of(p, cfg.tile_ex, cfg.tile_ez, &ntx, &ntz);
      rc = get_lists(p, cfg.tile_ex, cfg.tile_ez, &L);
    }
    if (rc) return rc;
    if (groups.empty() || groups.back().N != p->npol)
      groups.push_back(Group{p->npol, (long long)b->h_cta.size(), 0, false, false});
    Group& G = groups.back();
    G.adj |= (s.flags & SEM_F_ADJOINT) != 0;
    G.stc |= p->bnd_n > 0;
    char* a = b->arena + off;
    base[i] = off;
    SolveDev& d = b->h_solves[oi];
    d.nelx = p->nelx; d.nelz = p->nelz; d.nxg = p->nxg; d.nzg = p->nzg; d.pitch = p->pitch;
    d.tiles_x = ntx; d.tiles_z = ntz;
    d.zchunk = use_strip ? zchunk : p->nelz;
    d.tile_base = (int)(b->h_cta.size() - G.cta0);
    d.nt = p->nt; d.k = kk[i]; d.nseg = nseg[i]; d.flags = s.flags; d.start_tick = 0;
    d.it0 = s.it0; d.it1 = s.it1; d.decim = s.decim;
    d.src_gx = p->src_gx; d.src_gz = p->src_gz; d.nrec = p->nrec;
    d.fstride = p->fstride;
    d.c2 = (const float*)(a + ws[i].c2);
    d.W = (float*)(a + ws[i].W);
    d.V = (float*)(a + ws[i].V);
    d.ckpt = (s.flags & SEM_F_ADJOINT) ? (float*)(a + ws[i].ckpt) : nullptr;
    d.ring = (s.flags & SEM_F_ADJOINT) ? (float*)(a + ws[i].ring) : nullptr;
    d.L = (s.flags & SEM_F_ADJOINT) ? (float*)(a + ws[i].L) : nullptr;
    d.Mu = (s.flags & SEM_F_ADJOINT) ? (float*)(a + ws[i].Mu) : nullptr;
    d.grad = (s.flags & SEM_F_ADJOINT) ? (float*)(a + ws[i].grad) : nullptr;
    d.grad64 = (s.flags & SEM_F_ADJOINT) ? (double*)(a + ws[i].grad64) : nullptr;
    d.D = p->D; d.beta = p->beta; d.tx = p->tx; d.tz = p->tz; d.src_term = p->src_term;
    d.rec_base = p->rec_base; d.rec_w = p->rec_w;
    d.rec_tile_off = L.rec_off; d.rec_tile_ids = L.rec_ids;
    d.inj_tile_off = L.inj_off; d.inj_tile_ids = L.inj_ids;
    d.rec_out = s.rec_out; d.yobs = s.y_obs;
    d.misfit = (double*)(a + ws[i].misfit);
    d.rmax = d.misfit + p->nrec;
    d.adj_scale = d.misfit + 2 * p->nrec;
    d.status = (int*)(a + ws[i].status);
    d.ws = (const float*)a;
    d.tmap = nullptr;
    d.bnd_n = p->bnd_n; d.bnd_pitch = bnd_pitch_of(p);
    d.bnd_coef = p->bnd_n ? (const float*)(a + ws[i].bnd_coef) : nullptr;
    d.bnd_hist = ws[i].bnd_hist >= 0 ? (float*)(a + ws[i].bnd_hist) : nullptr;
    if (use_strip) {
      rc = encode_band_map(&b->h_tmaps[oi], a, p, field_slots(ws[i], p, s.flags & SEM_F_ADJOINT));
      if (rc) return rc;
      d.tmap = b->d_tmaps + oi;
    }
    for (int c = 0; c < ntiles; ++c) b->h_cta.push_back(oi - 0);
    G.ncta += ntiles;
    max_prog = std::max(max_prog, prog[i]);
    off += ws[i].bytes;
  }
  // cta map entries are indices into the group's descriptor sub-array
  for (auto& G : groups) {
    const int first = b->h_cta[G.cta0];
    for (long long c = G.cta0; c < G.cta0 + G.ncta; ++c) b->h_cta[c] -= first;
  }
  if (n > b->solves_cap) {
    cudaFree(b->d_solves);
    b->d_solves = nullptr;
    CUDA_TRY(cudaMalloc((void**)&b->d_solves, sizeof(SolveDev) * n));
    b->solves_cap = n;
  }
  if ((long long)b->h_cta.size() > b->cta_cap) {
    cudaFree(b->d_cta);
    b->d_cta = nullptr;
    CUDA_TRY(cudaMalloc((void**)&b->d_cta, sizeof(int) * b->h_cta.size()));
    b->cta_cap = b->h_cta.size();
  }
  CUDA_TRY(cudaMemcpyAsync(b->d_solves, b->h_solves.data(), sizeof(SolveDev) * n,
                           cudaMemcpyHostToDevice, stream));
  if (use_strip)
    CUDA_TRY(cudaMemcpyAsync(b->d_tmaps, b->h_tmaps.data(), sizeof(CUtensorMap) * n,
                             cudaMemcpyHostToDevice, stream));
  CUDA_TRY(cudaMemcpyAsync(b->d_cta, b->h_cta.data(), sizeof(int) * b->h_cta.size(),
                           cudaMemcpyHostToDevice, stream));

  // ---- per-solve inputs/outputs: one set-up launch (zero-start state, c^2) and one
  // output launch (gradient, log-likelihood, status) for the whole group
  b->h_io.assign(n, SolveIo{});
  long long max_pts = 1;
  for (int oi = 0; oi < n; ++oi) {
    const int i = order[oi];
    const sem_solve_t& s = solves[i];
    const sem_plan_s* p = s.plan;
    char* a = b->arena + base[i];
    const long long F = p->fstride * 4;
    SolveIo& io = b->h_io[oi];
    io.vel = s.velocity; io.pos = p->node_pos; io.c2 = (float*)(a + ws[i].c2);
    io.npoints = p->npoints;
    max_pts = std::max(max_pts, (long long)p->npoints);
    // zero initial state: b_0 (ckpt 0 or ring 0 or W 0), v_0 (ckpt 1 or V), adjoint state
    auto zero = [&](long long o, long long bytes) { io.zp[io.nzero] = a + o; io.zb[io.nzero++] = bytes; };
    zero(ws[i].W, F);
    zero(ws[i].V, F);
    if (s.flags & SEM_F_ADJOINT) {
      zero(ws[i].ckpt, 2 * F);
      zero(ws[i].ring, F);
      zero(ws[i].L, 3 * F);      // L[0], L[1], Mu
      zero(ws[i].grad, 3 * F);   // float32 partial and float64 accumulator
    }
    zero(ws[i].misfit, ws[i].status - ws[i].misfit + 256);
    if (ws[i].bnd_hist >= 0) zero(ws[i].bnd_hist, (long long)bnd_pitch_of(p) * 4);  // b_0 = 0
    io.bnd_n = p->bnd_n; io.bnd_pitch = bnd_pitch_of(p);
    io.bnd_ref = p->bnd_ref; io.bnd_alpha = p->bnd_alpha; io.bnd_gamma = p->bnd_gamma;
    io.bnd_coef = p->bnd_n ? (float*)(a + ws[i].bnd_coef) : nullptr;
    io.grad_out = ((s.flags & SEM_F_ADJOINT) && s.grad_out) ? s.grad_out : nullptr;
    io.gacc = (const double*)(a + ws[i].grad64);
    io.adj_scale = (const double*)(a + ws[i].misfit) + 2 * p->nrec;
    io.inv_sigma2 = s.inv_sigma2;
    io.misfit = (const double*)(a + ws[i].misfit);
    io.nrec = p->nrec;
    io.loglik_out = ((s.flags & SEM_F_MISFIT) && s.loglik_out) ? s.loglik_out : nullptr;
    io.st = (const int*)(a + ws[i].status);
    io.status_out = s.status_out;
  }
  if (n > b->io_cap) {
    cudaFree(b->d_io);
    b->d_io = nullptr;
    CUDA_TRY(cudaMalloc((void**)&b->d_io, sizeof(SolveIo) * n));
    b->io_cap = n;
  }
  CUDA_TRY(cudaMemcpyAsync(b->d_io, b->h_io.data(), sizeof(SolveIo) * n, cudaMemcpyHostToDevice, stream));
  const unsigned io_bx = (unsigned)std::min<long long>(64, (max_pts + 2047) / 2048);
  for (int s0 = 0; s0 < n; s0 += 65535) {
    batch_setup_kernel<<<dim3(io_bx, (unsigned)std::min(65535, n - s0)), 256, 0, stream>>>(b->d_io, s0);
    b->last_launches++;
  }
  CUDA_TRY(cudaMemsetAsync(b->d_tick, 0, sizeof(int), stream));
  CUDA_TRY(cudaGetLastError());

  // ---- per-group launch parameters
  struct Launch { KernelFn fn; long long cta0, ncta; size_t smem; int N; };
  std::vector<Launch> launches;
  for (auto& G : groups) {
    KernelFn fn = use_strip ? strip_kernel_for(G.N) : kernel_for(G.N);
    if (!fn) return fail(SEM_ERR_UNSUPPORTED, "polynomial order");
    const size_t smem = (size_t)(use_strip ? strip_smem_floats(G.N, G.adj) + (G.stc ? kStripBndFloats : 0)
                                           : smem_floats(G.N, cfg.tile_ex, cfg.tile_ez, G.adj)) *
                        sizeof(float);
    if (smem > 227 * 1024) return fail(SEM_ERR_ARG, "tile too large for shared memory");
    CUDA_TRY(raise_smem_limit((const void*)fn, smem));
    launches.push_back(Launch{fn, G.cta0, G.ncta, smem, G.N});
  }
  // solve descriptor sub-array of each group starts at the first solve of that group
  std::vector<const SolveDev*> gdesc;
  {
    int oi = 0;
    for (auto& G : groups) {
      gdesc.push_back(b->d_solves + oi);
      while (oi < n && solves[order[oi]].plan->npol == G.N) ++oi;
    }
  }
  // captured chunks replay with a device tick counter; plain launches pass the tick and
  // chain through programmatic dependent launch (no counter kernel between ticks)
  auto launch_tick = [&]() -> int {
    for (size_t gi = 0; gi < launches.size(); ++gi) {
      const Launch& Lc = launches[gi];
      Lc.fn<<<(unsigned)Lc.ncta, use_strip ? strip_threads(Lc.N) : cfg.threads, Lc.smem, stream>>>(
          gdesc[gi], b->d_cta + Lc.cta0, b->d_tick, cfg.tile_ex, cfg.tile_ez, 0);
    }
    tick_advance_kernel<<<1, 1, 0, stream>>>(b->d_tick);
    return SEM_OK;
  };
  auto launch_tick_pdl = [&](int tick) -> cudaError_t {
    for (size_t gi = 0; gi < launches.size(); ++gi) {
      const Launch& Lc = launches[gi];
      cudaLaunchConfig_t lc = {};
      lc.gridDim = dim3((unsigned)Lc.ncta);
      lc.blockDim = dim3(use_strip ? strip_threads(Lc.N) : cfg.threads);
      lc.dynamicSmemBytes = Lc.smem;
      lc.stream = stream;
      cudaLaunchAttribute at[1];
      at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
      at[0].val.programmaticStreamSerializationAllowed = SEM_PDL ? 1 : 0;
      lc.attrs = at;
      lc.numAttrs = 1;
      const int* no_counter = nullptr;
      cudaError_t e = cudaLaunchKernelEx(&lc, Lc.fn, gdesc[gi], (const int*)(b->d_cta + Lc.cta0),
                                         no_counter, cfg.tile_ex, cfg.tile_ez, tick);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  };

  // ---- the tick loop: plain launches or captured chunks, bracketed by events
  while ((int)b->tick_ev.size() < b->tick_ev_used + 2) {
    cudaEvent_t e;
    CUDA_TRY(cudaEventCreate(&e));
    b->tick_ev.push_back(e);
  }
  cudaEvent_t ev_begin = b->tick_ev[b->tick_ev_used], ev_end = b->tick_ev[b->tick_ev_used + 1];
  CUDA_TRY(cudaEventRecord(ev_begin, stream));
  const long long per_tick = (long long)launches.size() + 1;  // graphed: + counter kernel
  bool graphed = false, persisted = false;
  // persistent kernel: one cooperative launch for the whole tick program, when the group
  // has one polynomial order and all its CTAs are resident at once (else per-tick launches)
  if (cfg.kernel == 3 && launches.size() == 1) {
    const Launch& Lc = launches[0];
    PersistFn pf = persist_kernel_for(Lc.N);
    int nb = 0;
    if (pf && raise_smem_limit((const void*)pf, Lc.smem) == cudaSuccess &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, pf, cfg.threads, Lc.smem) == cudaSuccess &&
        (long long)nb * sms >= Lc.ncta) {
      unsigned long long* bar =
          reinterpret_cast<unsigned long long*>(reinterpret_cast<char*>(b->d_tick) + 128);
      CUDA_TRY(cudaMemsetAsync(bar, 0, sizeof(unsigned long long), stream));
      cudaLaunchConfig_t lc = {};
      lc.gridDim = dim3((unsigned)Lc.ncta);
      lc.blockDim = dim3(cfg.threads);
      lc.dynamicSmemBytes = Lc.smem;
      lc.stream = stream;
      cudaLaunchAttribute at[1];
      at[0].id = cudaLaunchAttributeCooperative;
      at[0].val.cooperative = 1;
      lc.attrs = at;
      lc.numAttrs = 1;
      CUDA_TRY(cudaLaunchKernelEx(&lc, pf, gdesc[0], (const int*)(b->d_cta + Lc.cta0), 0, max_prog,
                                  cfg.tile_ex, cfg.tile_ez, bar));
      b->last_launches += 1;
      persisted = true;
    }
    cudaGetLastError();  // a refused occupancy query leaves the per-tick path
  }
  // persistent strip kernel: one cooperative launch over every chunk of a one-order group,
  // when all of them are resident at once (else per-tick strip launches)
  if (cfg.kernel == 4 && use_strip && launches.size() == 1) {
    const Launch& Lc = launches[0];
    StripPersistFn pf = strip_persist_kernel_for(Lc.N);
    int nb = 0;
    const long long sync_bytes = round_up(Lc.ncta * 4, 256) + round_up((long long)n * 8, 256);
    if (pf && raise_smem_limit((const void*)pf, Lc.smem) == cudaSuccess &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, pf, strip_threads(Lc.N), Lc.smem) == cudaSuccess &&
        (long long)nb * sms >= Lc.ncta) {
      if (sync_bytes > b->sync_cap) {
        cudaFree(b->d_sync);
        b->d_sync = nullptr;
        b->sync_cap = 0;
        CUDA_TRY(cudaMalloc((void**)&b->d_sync, sync_bytes));
        b->sync_cap = sync_bytes;
      }
      CUDA_TRY(cudaMemsetAsync(b->d_sync, 0, sync_bytes, stream));
      unsigned* done = reinterpret_cast<unsigned*>(b->d_sync);
      unsigned long long* sbar =
          reinterpret_cast<unsigned long long*>(b->d_sync + round_up(Lc.ncta * 4, 256));
      cudaLaunchConfig_t lc = {};
      lc.gridDim = dim3((unsigned)Lc.ncta);
      lc.blockDim = dim3(strip_threads(Lc.N));
      lc.dynamicSmemBytes = Lc.smem;
      lc.stream = stream;
      cudaLaunchAttribute at[1];
      at[0].id = cudaLaunchAttributeCooperative;
      at[0].val.cooperative = 1;
      lc.attrs = at;
      lc.numAttrs = 1;
      CUDA_TRY(cudaLaunchKernelEx(&lc, pf, gdesc[0], (const int*)(b->d_cta + Lc.cta0), 0, max_prog, done, sbar));
      b->last_launches += 1;
      persisted = true;
      b->last_kernel = 4;
    }
    cudaGetLastError();  // a refused occupancy query leaves the per-tick path
  }
  b->last_kernel = (persisted && b->last_kernel != 4) ? 3 : b->last_kernel;
  if (!persisted && cfg.graph_chunk > 0 && stream != nullptr && stream != cudaStreamLegacy &&
      stream != cudaStreamPerThread) {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    const int chunk = std::min(cfg.graph_chunk, max_prog);
    if (cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
      for (int c = 0; c < chunk; ++c) launch_tick();
      cudaError_t e = cudaStreamEndCapture(stream, &graph);
      if (e == cudaSuccess && cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess) {
        const int reps = (max_prog + chunk - 1) / chunk;
        for (int r = 0; r < reps; ++r) CUDA_TRY(cudaGraphLaunch(exec, stream));
        b->last_launches += (long long)reps * chunk * per_tick;
        graphed = true;
      }
      if (exec) cudaGraphExecDestroy(exec);
      if (graph) cudaGraphDestroy(graph);
    }
    cudaGetLastError();  // clear a failed capture
  }
  if (!graphed && !persisted) {
    for (int tick = 0; tick < max_prog; ++tick) CUDA_TRY(launch_tick_pdl(tick));
    b->last_launches += (long long)max_prog * (long long)launches.size();
  }
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaEventRecord(ev_end, stream));
  b->tick_ev_used += 2;
  b->last_ticks += max_prog;

  // ---- outputs
  for (int s0 = 0; s0 < n; s0 += 65535) {
    batch_output_kernel<<<dim3(io_bx, (unsigned)std::min(65535, n - s0)), 256, 0, stream>>>(b->d_io, s0);
    b->last_launches++;
  }
  CUDA_TRY(cudaGetLastError());
  return SEM_OK;
}

namespace {

// Time of one tick in units of the per-CTA work: CTAs beyond one resident wave queue
// behind it, and each round costs a fixed latency part plus a part growing with the
// CTAs resident per SM (the strip kernel's tick times fit 6.4 + CTAs/SM).
double tick_rounds(long long ctas, long long slots, int sms) {
  double c = 0.0;
  for (long long left = ctas; left > 0; left -= slots)
    c += 6.4 + (double)std::min(left, slots) / sms;
  return c;
}

struct GroupPlan { int begin, end, k; };

// Automatic schedule for solves with ckpt_k = 0: split the batch (in the caller's order)
// into g consecutive groups of equal size run one after another, each with the largest
// checkpoint interval whose workspace fits the memory budget (k = nt: no replay), and
// pick the g with the smallest modelled time.  Explicit ckpt_k values are kept.
int auto_schedule(const sem_solve_t* sv, int n, const sem_launch_cfg_t& cfg, long long budget,
                  std::vector<GroupPlan>* out) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // per-solve CTAs of either kernel and resident CTAs per SM (first solve's order)
  std::vector<long long> strips(n), tiles(n);
  for (int i = 0; i < n; ++i) {
    const sem_plan_s* p = sv[i].plan;
    strips[i] = strips_of(p, nullptr);
    int tx, tz;
    tiles[i] = tiles_of(p, cfg.tile_ex, cfg.tile_ez, &tx, &tz);
  }
  bool any_adj = false, any_stc = false;
  for (int i = 0; i < n; ++i) any_adj |= (sv[i].flags & SEM_F_ADJOINT) != 0;
  for (int i = 0; i < n; ++i) any_stc |= sv[i].plan->bnd_n > 0;
  const int N0 = sv[0].plan->npol;
  auto occupancy = [&](bool strip) -> long long {
    KernelFn fn = strip ? strip_kernel_for(N0) : kernel_for(N0);
    const size_t smem = (size_t)(strip ? strip_smem_floats(N0, any_adj) + (any_stc ? kStripBndFloats : 0)
                                       : smem_floats(N0, cfg.tile_ex, cfg.tile_ez, any_adj)) * 4;
    int nb = 1;
    if (smem <= 227 * 1024 &&
        raise_smem_limit((const void*)fn, smem) == cudaSuccess &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, strip ? strip_threads(N0) : cfg.threads, smem) ==
            cudaSuccess)
      nb = std::max(nb, 1);
    else
      nb = 1;
    cudaGetLastError();
    return (long long)nb * sms;
  };
  const long long slots_strip = occupancy(true), slots_tile = occupancy(false);

  double best = -1.0;
  std::vector<GroupPlan> best_plan;
  const int gmax = std::min(n, 64);
  for (int g = 1; g <= gmax; ++g) {
    const int m = (n + g - 1) / g;
    std::vector<GroupPlan> plan;
    double cost = 0.0;
    bool ok = true;
    for (int b0 = 0; b0 < n && ok; b0 += m) {
      const int b1 = std::min(n, b0 + m);
      // largest common k for the automatic solves whose workspaces fit the budget
      int nt_max = 2, k_floor = 2;
      for (int i = b0; i < b1; ++i)
        if ((sv[i].flags & SEM_F_ADJOINT) && sv[i].ckpt_k <= 0) {
          nt_max = std::max(nt_max, sv[i].plan->nt);
          k_floor = std::max(k_floor, std::min(sv[i].plan->nt, (int)std::sqrt(2.0 * sv[i].plan->nt)));
        }
      auto bytes_at = [&](int k) {
        long long tot = 0;
        int ns;
        for (int i = b0; i < b1; ++i) {
          const bool adj = sv[i].flags & SEM_F_ADJOINT;
          const int ki = !adj ? 2 : (sv[i].ckpt_k > 0 ? sv[i].ckpt_k : std::min(k, sv[i].plan->nt));
          tot += layout(sv[i].plan, sv[i].flags, std::max(2, std::min(ki, sv[i].plan->nt)), &ns).bytes;
        }
        return tot;
      };
      if (bytes_at(k_floor) > budget) { ok = false; break; }
      int lo = k_floor, hi = nt_max;
      while (lo < hi) {
        const int mid = lo + (hi - lo + 1) / 2;
        if (bytes_at(mid) <= budget) lo = mid; else hi = mid - 1;
      }
      const int k = lo;
      // modelled time: forward-like ticks (forward + replay) and adjoint ticks (x1.5)
      long long fwd_ticks = 0, adj_ticks = 0, nstrip = 0, ntile = 0, nchunk_min = 0;
      int nelz_max = 1;
      for (int i = b0; i < b1; ++i) {
        const sem_solve_t& s = sv[i];
        const int nt = s.plan->nt;
        const bool adj = s.flags & SEM_F_ADJOINT;
        const int ki = std::max(2, std::min(adj ? (s.ckpt_k > 0 ? s.ckpt_k : k) : 2, nt));
        const int nseg = (nt + ki - 1) / ki;
        fwd_ticks = std::max(fwd_ticks, (long long)nt + 1 + (adj ? (long long)ki * (nseg - 1) : 0));
        if (adj) adj_ticks = std::max(adj_ticks, (long long)nt);
        nstrip += strips[i];
        ntile += tiles[i];
        nchunk_min += strips[i] * ((s.plan->nelz + kMinChunk - 1) / kMinChunk);
        nelz_max = std::max(nelz_max, s.plan->nelz);
      }
      const bool strip = cfg.kernel == 2 || cfg.kernel == 4 || (cfg.kernel == 0 && strip_fills(nchunk_min, sms));
      long long nstrip_ctas = 0;
      if (strip) {
        const int zc = strip_zchunk(nstrip, nelz_max, sms, cfg.strip_bands);
        for (int i = b0; i < b1; ++i) nstrip_ctas += strips[i] * ((sv[i].plan->nelz + zc - 1) / zc);
      }
      const double per_tick = strip ? tick_rounds(nstrip_ctas, slots_strip, sms) : tick_rounds(ntile, slots_tile, sms);
      cost += per_tick * ((double)fwd_ticks + 1.5 * (double)adj_ticks);
      plan.push_back(GroupPlan{b0, b1, k});
    }
    if (!ok) continue;
    if (best < 0.0 || cost < 0.98 * best) { best = cost; best_plan = plan; }
  }
  if (best < 0.0) {  // nothing fits: one solve at a time with the smallest workspace
    for (int i = 0; i < n; ++i) {
      const int nt = sv[i].plan->nt;
      best_plan.push_back(GroupPlan{i, i + 1, std::max(2, std::min(nt, (int)std::sqrt(2.0 * nt)))});
    }
  }
  *out = best_plan;
  return SEM_OK;
}

}  // namespace

extern "C" {

int sem_run(sem_batch_t* b, const sem_solve_t* solves, int32_t n, const sem_launch_cfg_t* cfg_in,
            void* stream_v) {
  if (!b || (!solves && n) || n < 0) return fail(SEM_ERR_ARG, "null argument");
  cudaStream_t stream = (cudaStream_t)stream_v;
  // no configuration: automatic kernel, tile shape, strip chunks and memory budget
  sem_launch_cfg_t cfg = cfg_in ? *cfg_in : sem_launch_cfg_t{0, 0, 256, 0, 0, 0, 0};
  if (!(cfg.tile_ex == 0 && cfg.tile_ez == 0) && (cfg.tile_ex < 1 || cfg.tile_ez < 1))
    return fail(SEM_ERR_ARG, "tile size must be >= 1 (or 0 x 0: automatic)");
  if (cfg.kernel < 0 || cfg.kernel > 4)
    return fail(SEM_ERR_ARG,
                "kernel must be 0 (auto), 1 (tile), 2 (strip), 3 (persistent tile), 4 (persistent strip)");
  if (cfg.threads < 32 || cfg.threads > 256 || cfg.threads % 32) cfg.threads = 256;
  if (cfg.memory_budget < 0) return fail(SEM_ERR_ARG, "memory_budget must be >= 0");
  if (cfg.strip_bands < 0) return fail(SEM_ERR_ARG, "strip_bands must be >= 0");
  b->last_launches = 0;
  b->last_groups = 0;
  b->last_ticks = 0;
  b->tick_ev_used = 0;
  if (n == 0) return SEM_OK;
  bool any_auto = false;
  for (int i = 0; i < n; ++i) {
    if (!solves[i].plan) return fail(SEM_ERR_ARG, "solve missing plan/velocity/rec_out");
    any_auto |= (solves[i].flags & SEM_F_ADJOINT) && solves[i].ckpt_k <= 0;
  }
  if (cfg.tile_ex == 0) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    auto_tile(solves, n, sms, cfg.threads, &cfg.tile_ex, &cfg.tile_ez);
  }
  b->last_tile_ex = cfg.tile_ex;
  b->last_tile_ez = cfg.tile_ez;
  if (!any_auto) {
    b->last_groups = 1;
    return run_group(b, solves, n, cfg, stream);
  }
  long long budget = cfg.memory_budget;
  if (budget == 0) {
    size_t fr = 0, tot = 0;
    CUDA_TRY(cudaMemGetInfo(&fr, &tot));
    budget = (long long)(0.85 * (double)((long long)fr + b->arena_bytes)) - (512LL << 20);
    budget = std::max(budget, 1LL << 20);
  }
  std::vector<GroupPlan> groups;
  int rc = auto_schedule(solves, n, cfg, budget, &groups);
  if (rc) return rc;
  std::vector<sem_solve_t> sv(solves, solves + n);
  for (const GroupPlan& g : groups) {
    for (int i = g.begin; i < g.end; ++i)
      if ((sv[i].flags & SEM_F_ADJOINT) && sv[i].ckpt_k <= 0) sv[i].ckpt_k = g.k;
    rc = run_group(b, sv.data() + g.begin, g.end - g.begin, cfg, stream);
    if (rc) return rc;
    b->last_groups++;
  }
  return SEM_OK;
}

int32_t sem_batch_last_groups(const sem_batch_t* b) { return b ? b->last_groups : -1; }

int sem_batch_last_shape(const sem_batch_t* b, int32_t* tile_ex, int32_t* tile_ez, int32_t* strip_bands) {
  if (!b) return fail(SEM_ERR_ARG, "null argument");
  if (tile_ex) *tile_ex = b->last_tile_ex;
  if (tile_ez) *tile_ez = b->last_tile_ez;
  if (strip_bands) *strip_bands = b->last_zchunk;
  return SEM_OK;
}

int64_t sem_batch_last_ticks(const sem_batch_t* b) { return b ? b->last_ticks : -1; }

int sem_batch_last_tick_ms(const sem_batch_t* b, double* ms_out) {
  if (!b || !ms_out) return fail(SEM_ERR_ARG, "null argument");
  double tot = 0.0;
  for (int i = 0; i + 1 < b->tick_ev_used; i += 2) {
    CUDA_TRY(cudaEventSynchronize(b->tick_ev[i + 1]));
    float ms = 0.f;
    CUDA_TRY(cudaEventElapsedTime(&ms, b->tick_ev[i], b->tick_ev[i + 1]));
    tot += ms;
  }
  *ms_out = tot;
  return SEM_OK;
}

int sem_selftest_wait(int32_t which, int32_t* status_out) {
  if (!status_out || which < 0 || which > 2) return fail(SEM_ERR_ARG, "which must be 0, 1 or 2");
  char* buf = nullptr;
  CUDA_TRY(cudaMalloc((void**)&buf, 256));
  int rc = SEM_OK;
  unsigned long long* bar = reinterpret_cast<unsigned long long*>(buf);
  int* st = reinterpret_cast<int*>(buf + 128);
  cudaError_t e = cudaMemset(buf, 0, 256);
  if (e == cudaSuccess) {
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3(which == 0 ? 1u : 2u);
    lc.blockDim = dim3(32);
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    lc.attrs = at;
    lc.numAttrs = which == 0 ? 0 : 1;
    e = cudaLaunchKernelEx(&lc, wait_probe_kernel, (int)which, bar, st);
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  int h = 0;
  if (e == cudaSuccess) e = cudaMemcpy(&h, st, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) rc = fail(SEM_ERR_CUDA, cudaGetErrorString(e));
  cudaFree(buf);
  *status_out = h;
  return rc;
}

int sem_forward_noalloc(const sem_plan_t* p, const double* velocity, float* rec_out,
                        int32_t* status_out, void* stream_v) {
  if (!p || !velocity || !rec_out) return fail(SEM_ERR_ARG, "null argument");
  cudaStream_t stream = (cudaStream_t)stream_v;
  int dev = -1;
  CUDA_TRY(cudaGetDevice(&dev));
  if (dev != p->device) return fail(SEM_ERR_ARG, "plan was created on another device");
  if (p->bnd_n > 0)
    return fail(SEM_ERR_UNSUPPORTED, "sem_forward_noalloc runs the sponge boundary mode only");
  // device address of the scratch array on this device, looked up when the plan was made
  char* const base = p->noalloc_scratch;
  if (!base) return fail(SEM_ERR_ARG, "plan has no scratch address");
  // receiver lists of the default tiles were built when the plan was created
  sem_plan_s::Lists L{};
  {
    std::lock_guard<std::mutex> lk(p->mu);
    auto it = p->lists.find(std::make_pair(kNoAllocTile, kNoAllocTile));
    if (it == p->lists.end()) return fail(SEM_ERR_ARG, "plan has no default tile lists");
    L = it->second;
  }
  int ntx, ntz;
  const int ntiles = tiles_of(p, kNoAllocTile, kNoAllocTile, &ntx, &ntz);
  // scratch layout: descriptor | tick | CTA map | c^2 | b[2] | v | misfit block | status
  const long long F = p->fstride * 4;
  long long o = 0;
  const long long o_desc = o; o += round_up(sizeof(SolveDev), 256);
  const long long o_tick = o; o += 256;
  const long long o_cta = o; o += round_up((long long)ntiles * 4, 256);
  const long long o_c2 = o; o += F;
  const long long o_W = o; o += 2 * F;
  const long long o_V = o; o += F;
  const long long o_mis = o; o += round_up((long long)(2 * p->nrec + 1) * 8, 256);
  const long long o_st = o; o += 256;
  if (o > (long long)kNoAllocScratchBytes)
    return fail(SEM_ERR_ARG, "mesh too large for sem_forward_noalloc: needs " + std::to_string(o) +
                                 " bytes of scratch, the limit is " + std::to_string(kNoAllocScratchBytes));
  SolveDev d{};
  d.nelx = p->nelx; d.nelz = p->nelz; d.nxg = p->nxg; d.nzg = p->nzg; d.pitch = p->pitch;
  d.tiles_x = ntx; d.tiles_z = ntz; d.tile_base = 0;
  d.zchunk = p->nelz;
  d.nt = p->nt; d.k = 2; d.nseg = 1; d.flags = 0; d.start_tick = 0;
  d.it0 = 0; d.it1 = p->nt; d.decim = 1;
  d.src_gx = p->src_gx; d.src_gz = p->src_gz; d.nrec = p->nrec;
  d.fstride = p->fstride;
  d.c2 = (const float*)(base + o_c2);
  d.W = (float*)(base + o_W);
  d.V = (float*)(base + o_V);
  d.D = p->D; d.beta = p->beta; d.tx = p->tx; d.tz = p->tz; d.src_term = p->src_term;
  d.rec_base = p->rec_base; d.rec_w = p->rec_w;
  d.rec_tile_off = L.rec_off; d.rec_tile_ids = L.rec_ids;
  d.inj_tile_off = L.inj_off; d.inj_tile_ids = L.inj_ids;
  d.rec_out = rec_out; d.yobs = nullptr;
  d.misfit = (double*)(base + o_mis);
  d.rmax = d.misfit + p->nrec;
  d.adj_scale = d.misfit + 2 * p->nrec;
  d.status = (int*)(base + o_st);
  // b_0 = 0 and v_0 = 0: W[0] (first state) and V; the previous call left its state here
  noalloc_setup_kernel<<<256, 256, 0, stream>>>(d, (SolveDev*)(base + o_desc), (int*)(base + o_cta), ntiles,
                                                (int*)(base + o_tick), (float*)(base + o_W),
                                                3 * p->fstride, (int*)(base + o_st));
  set_c2_kernel<<<std::min(1024, (p->npoints + 255) / 256), 256, 0, stream>>>(
      velocity, p->node_pos, (float*)(base + o_c2), p->npoints);
  KernelFn fn = kernel_for(p->npol);
  const size_t smem = (size_t)smem_floats(p->npol, kNoAllocTile, kNoAllocTile, false) * sizeof(float);
  CUDA_TRY(raise_smem_limit((const void*)fn, smem));
  // ticks: the tick number is an argument and consecutive ticks chain by programmatic
  // dependent launch, as on sem_run's plain-launch path
  for (int tick = 0; tick < p->nt; ++tick) {
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3((unsigned)ntiles);
    lc.blockDim = dim3(256);
    lc.dynamicSmemBytes = smem;
    lc.stream = stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = SEM_PDL ? 1 : 0;
    lc.attrs = at;
    lc.numAttrs = 1;
    const int* no_counter = nullptr;
    CUDA_TRY(cudaLaunchKernelEx(&lc, fn, (const SolveDev*)(base + o_desc), (const int*)(base + o_cta),
                                no_counter, kNoAllocTile, kNoAllocTile, tick));
  }
  if (status_out) copy_status_kernel<<<1, 32, 0, stream>>>((const int*)(base + o_st), status_out);
  CUDA_TRY(cudaGetLastError());
  return SEM_OK;
}

int sem_forward(sem_batch_t* b, const sem_plan_t* plan, const double* velocity, float* rec_out,
                void* stream) {
  if (!plan) return fail(SEM_ERR_ARG, "null plan");
  sem_solve_t s{};
  s.plan = plan; s.velocity = velocity; s.flags = 0; s.ckpt_k = 2;
  s.it0 = 0; s.it1 = plan->nt; s.decim = 1; s.rec_out = rec_out;
  return sem_run(b, &s, 1, nullptr, stream);
}

int sem_forward_adjoint(sem_batch_t* b, const sem_plan_t* plan, const double* velocity,
                        const double* y_obs, double inv_sigma2, int32_t exact, int32_t ckpt_k,
                        float* clean_out, double* loglik_out, double* grad_out, void* stream) {
  if (!plan) return fail(SEM_ERR_ARG, "null plan");
  sem_solve_t s{};
  s.plan = plan; s.velocity = velocity;
  s.flags = SEM_F_ADJOINT | SEM_F_MISFIT | SEM_F_SHIFT | (exact ? SEM_F_EXACT : 0);
  s.ckpt_k = ckpt_k; s.y_obs = y_obs; s.it0 = 0; s.it1 = plan->nt; s.decim = 1;
  s.inv_sigma2 = inv_sigma2; s.rec_out = clean_out; s.loglik_out = loglik_out; s.grad_out = grad_out;
  return sem_run(b, &s, 1, nullptr, stream);
}

}  // extern "C"

// ============================================================================
// serving engine: continuous batching over the tick program
// ============================================================================
struct EngineJob {
  sem_solve_t s{};
  int64_t ticket = 0;
  int k = 2, nseg = 1, prog = 0, ntiles = 0, state = 0;  // 0 queued, 1 running, 2 retired
  long long start = 0, off = -1;
  Workspace ws{};
  cudaEvent_t ev = nullptr;
  CUtensorMap tmap{};     // strip kernel: band-load map of its workspace (fixed while running)
  bool has_tmap = false;
};

struct sem_engine_s {
  sem_engine_cfg_t cfg{};
  int device = -1;
  char* arena = nullptr;
  long long arena_bytes = 0;
  std::map<long long, long long> free_;  // offset -> size (first fit, coalesced)
  long long in_use = 0;
  int* d_tick = nullptr;
  long long tick = 0;
  SolveDev* d_solves = nullptr;
  int solves_cap = 0;
  int* d_cta = nullptr;
  long long cta_cap = 0;
  std::deque<EngineJob*> queue;
  std::vector<EngineJob*> running;
  std::map<int64_t, EngineJob*> jobs;
  int64_t next_ticket = 1;
  long long launches = 0;
  std::vector<SolveDev> h_solves;
  std::vector<int> h_cta;
  SolveIo* d_io = nullptr;  // [2 * max_solves]: outputs of retiring solves | set-up of admitted
  std::vector<SolveIo> h_io;
  CUtensorMap* d_tmaps = nullptr;
  int tmaps_cap = 0;
  std::vector<CUtensorMap> h_tmaps;
};

namespace {

// set-up / output table entry of one solve whose workspace starts at `a`
SolveIo solve_io(const sem_solve_t& s, const Workspace& ws, char* a) {
  const sem_plan_s* p = s.plan;
  const long long F = p->fstride * 4;
  SolveIo io{};
  io.vel = s.velocity; io.pos = p->node_pos; io.c2 = (float*)(a + ws.c2);
  io.npoints = p->npoints;
  auto zero = [&](long long o, long long bytes) { io.zp[io.nzero] = a + o; io.zb[io.nzero++] = bytes; };
  zero(ws.W, F);
  zero(ws.V, F);
  if (s.flags & SEM_F_ADJOINT) {
    zero(ws.ckpt, 2 * F);
    zero(ws.ring, F);
    zero(ws.L, 3 * F);  // L[0], L[1], Mu
    zero(ws.grad, 3 * F);  // float32 partial and float64 accumulator
  }
  zero(ws.misfit, ws.status - ws.misfit + 256);
  if (ws.bnd_hist >= 0) zero(ws.bnd_hist, (long long)bnd_pitch_of(p) * 4);  // b_0 = 0
  io.bnd_n = p->bnd_n; io.bnd_pitch = bnd_pitch_of(p);
  io.bnd_ref = p->bnd_ref; io.bnd_alpha = p->bnd_alpha; io.bnd_gamma = p->bnd_gamma;
  io.bnd_coef = p->bnd_n ? (float*)(a + ws.bnd_coef) : nullptr;
  io.grad_out = ((s.flags & SEM_F_ADJOINT) && s.grad_out) ? s.grad_out : nullptr;
  io.gacc = (const double*)(a + ws.grad64);
  io.adj_scale = (const double*)(a + ws.misfit) + 2 * p->nrec;
  io.inv_sigma2 = s.inv_sigma2;
  io.misfit = (const double*)(a + ws.misfit);
  io.nrec = p->nrec;
  io.loglik_out = ((s.flags & SEM_F_MISFIT) && s.loglik_out) ? s.loglik_out : nullptr;
  io.st = (const int*)(a + ws.status);
  io.status_out = s.status_out;
  return io;
}

long long arena_alloc(sem_engine_s* e, long long bytes) {
  bytes = round_up(bytes, 256);
  for (auto it = e->free_.begin(); it != e->free_.end(); ++it) {
    if (it->second >= bytes) {
      const long long off = it->first, rest = it->second - bytes;
      e->free_.erase(it);
      if (rest > 0) e->free_[off + bytes] = rest;
      e->in_use += bytes;
      return off;
    }
  }
  return -1;
}

void arena_free(sem_engine_s* e, long long off, long long bytes) {
  bytes = round_up(bytes, 256);
  e->in_use -= bytes;
  auto it = e->free_.emplace(off, bytes).first;
  auto nx = std::next(it);
  if (nx != e->free_.end() && it->first + it->second == nx->first) {
    it->second += nx->second;
    e->free_.erase(nx);
  }
  if (it != e->free_.begin()) {
    auto pv = std::prev(it);
    if (pv->first + pv->second == it->first) {
      pv->second += it->second;
      e->free_.erase(it);
    }
  }
}

}  // namespace

extern "C" {

int sem_engine_create(const sem_engine_cfg_t* cfg, sem_engine_t** out) {
  if (!cfg || !out) return fail(SEM_ERR_ARG, "null argument");
  if (cfg->max_solves < 1 || cfg->memory_cap < (1 << 20) || cfg->ticks_per_step < 1 ||
      cfg->kernel < 0 || cfg->kernel > 2 ||
      (!(cfg->tile_ex == 0 && cfg->tile_ez == 0) && (cfg->tile_ex < 1 || cfg->tile_ez < 1)))
    return fail(SEM_ERR_ARG, "bad engine configuration");
  auto* e = new sem_engine_s();
  e->cfg = *cfg;
  cudaGetDevice(&e->device);
  cudaError_t err = cudaMalloc((void**)&e->arena, cfg->memory_cap);
  if (err != cudaSuccess) {
    delete e;
    return fail(SEM_ERR_OOM, std::string("engine arena: ") + cudaGetErrorString(err));
  }
  e->arena_bytes = cfg->memory_cap;
  e->free_[0] = cfg->memory_cap;
  if (cudaMalloc((void**)&e->d_tick, 256) != cudaSuccess ||
      cudaMemset(e->d_tick, 0, sizeof(int)) != cudaSuccess) {
    cudaFree(e->arena);
    delete e;
    return fail(SEM_ERR_OOM, "engine tick counter");
  }
  *out = e;
  return SEM_OK;
}

int sem_engine_destroy(sem_engine_t* e) {
  if (!e) return SEM_OK;
  cudaDeviceSynchronize();
  for (auto& kv : e->jobs) {
    if (kv.second->ev) cudaEventDestroy(kv.second->ev);
    delete kv.second;
  }
  cudaFree(e->arena); cudaFree(e->d_tick); cudaFree(e->d_solves); cudaFree(e->d_cta); cudaFree(e->d_tmaps);
  cudaFree(e->d_io);
  delete e;
  return SEM_OK;
}

int sem_engine_submit(sem_engine_t* e, const sem_solve_t* s, int64_t* ticket) {
  if (!e || !s || !ticket) return fail(SEM_ERR_ARG, "null argument");
  if (!s->plan || !s->velocity || !s->rec_out) return fail(SEM_ERR_ARG, "solve missing plan/velocity/rec_out");
  const bool adj = s->flags & SEM_F_ADJOINT;
  if (adj && !(s->flags & SEM_F_SHIFT)) return fail(SEM_ERR_ARG, "adjoint requires the shifted receiver convention");
  if ((adj || (s->flags & SEM_F_MISFIT)) && !s->y_obs) return fail(SEM_ERR_ARG, "y_obs required");
  if (s->decim < 1 || s->it0 < 0 || s->it1 > s->plan->nt || s->it0 >= s->it1)
    return fail(SEM_ERR_ARG, "bad misfit window");
  if (s->plan->device != e->device) return fail(SEM_ERR_ARG, "plan and engine on different devices");
  auto* j = new EngineJob();
  j->s = *s;
  j->ticket = e->next_ticket++;
  j->k = adj ? std::max(2, std::min((int)s->ckpt_k, s->plan->nt)) : 2;
  j->ws = layout(s->plan, s->flags, j->k, &j->nseg);
  if (j->ws.bytes > e->arena_bytes) {
    delete j;
    return fail(SEM_ERR_ARG, "solve needs more device memory than the engine's cap");
  }
  const int nt = s->plan->nt;
  j->prog = nt + ((s->flags & SEM_F_SHIFT) ? 1 : 0) + (adj ? 1 + nt + j->k * (j->nseg - 1) : 0);
  e->queue.push_back(j);
  e->jobs[j->ticket] = j;
  *ticket = j->ticket;
  return SEM_OK;
}

int sem_engine_status(sem_engine_t* e, int64_t ticket, int32_t* state) {
  if (!e || !state) return fail(SEM_ERR_ARG, "null argument");
  auto it = e->jobs.find(ticket);
  if (it == e->jobs.end()) { *state = -1; return SEM_OK; }
  EngineJob* j = it->second;
  if (j->state < 2) { *state = j->state; return SEM_OK; }
  const cudaError_t q = cudaEventQuery(j->ev);
  if (q == cudaErrorNotReady) { *state = 1; return SEM_OK; }
  CUDA_TRY(q);
  *state = 2;
  return SEM_OK;
}

int sem_engine_release(sem_engine_t* e, int64_t ticket) {
  if (!e) return fail(SEM_ERR_ARG, "null argument");
  auto it = e->jobs.find(ticket);
  if (it == e->jobs.end()) return SEM_OK;
  EngineJob* j = it->second;
  if (j->state != 2) return fail(SEM_ERR_ARG, "solve still queued or running");
  if (j->ev) {
    CUDA_TRY(cudaEventSynchronize(j->ev));
    cudaEventDestroy(j->ev);
  }
  delete j;
  e->jobs.erase(it);
  return SEM_OK;
}

int sem_engine_stats(const sem_engine_t* e, int64_t* out) {
  if (!e || !out) return fail(SEM_ERR_ARG, "null argument");
  out[0] = (int64_t)e->queue.size();
  out[1] = (int64_t)e->running.size();
  out[2] = e->in_use;
  out[3] = e->tick;
  out[4] = e->launches;
  return SEM_OK;
}

int sem_engine_step(sem_engine_t* e, void* stream_v) {
  if (!e) return fail(SEM_ERR_ARG, "null argument");
  cudaStream_t stream = (cudaStream_t)stream_v;
  if (!e->d_io) {
    CUDA_TRY(cudaMalloc((void**)&e->d_io, sizeof(SolveIo) * 2 * (size_t)e->cfg.max_solves));
  }
  e->h_io.clear();
  // ---- retire solves whose program has ended: outputs (one launch), then free the workspace
  std::vector<EngineJob*> retiring;
  for (size_t i = 0; i < e->running.size();) {
    EngineJob* j = e->running[i];
    if (e->tick < j->start + j->prog) { ++i; continue; }
    e->h_io.push_back(solve_io(j->s, j->ws, e->arena + j->off));
    retiring.push_back(j);
    e->running.erase(e->running.begin() + i);
  }
  const int nret = (int)e->h_io.size();
  // ---- admit queued solves in arrival order while a slot and memory are free (their
  // workspaces may reuse the retiring solves' memory: the set-up launch follows the
  // output launch on the stream)
  for (EngineJob* j : retiring) arena_free(e, j->off, j->ws.bytes);
  std::vector<EngineJob*> admitted;
  while (!e->queue.empty() && (int)e->running.size() < e->cfg.max_solves) {
    EngineJob* j = e->queue.front();
    const long long off = arena_alloc(e, j->ws.bytes);
    if (off < 0) break;
    e->queue.pop_front();
    j->off = off;
    j->start = e->tick;
    j->state = 1;
    e->h_io.push_back(solve_io(j->s, j->ws, e->arena + off));
    admitted.push_back(j);
    e->running.push_back(j);
  }
  const int nadm = (int)e->h_io.size() - nret;
  if (!e->h_io.empty())
    CUDA_TRY(cudaMemcpyAsync(e->d_io, e->h_io.data(), sizeof(SolveIo) * e->h_io.size(),
                             cudaMemcpyHostToDevice, stream));
  auto io_blocks = [&](int s0, int cnt) {
    long long mx = 1;
    for (int i = s0; i < s0 + cnt; ++i) mx = std::max(mx, (long long)e->h_io[i].npoints);
    return (unsigned)std::min<long long>(64, (mx + 2047) / 2048);
  };
  if (nret > 0) {
    batch_output_kernel<<<dim3(io_blocks(0, nret), (unsigned)nret), 256, 0, stream>>>(e->d_io, 0);
    e->launches++;
    for (EngineJob* j : retiring) {
      CUDA_TRY(cudaEventCreateWithFlags(&j->ev, cudaEventDisableTiming));
      CUDA_TRY(cudaEventRecord(j->ev, stream));
      j->state = 2;
    }
  }
  if (nadm > 0) {
    batch_setup_kernel<<<dim3(io_blocks(nret, nadm), (unsigned)nadm), 256, 0, stream>>>(e->d_io, nret);
    e->launches++;
  }
  if (e->running.empty()) return SEM_OK;
  // ---- kernel and launch shape for the running set (as in sem_run: automatic variant,
  // strip chunks and tile shape unless the configuration fixes them)
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  std::vector<sem_solve_t> run_sv;
  long long total_strips = 0, min_chunk_ctas = 0;
  int nelz_max = 1;
  for (EngineJob* j : e->running) {
    run_sv.push_back(j->s);
    const sem_plan_s* p = j->s.plan;
    const int ns = strips_of(p, nullptr);
    total_strips += ns;
    min_chunk_ctas += (long long)ns * ((p->nelz + kMinChunk - 1) / kMinChunk);
    nelz_max = std::max(nelz_max, p->nelz);
  }
  const bool use_strip = e->cfg.kernel == 2 || (e->cfg.kernel == 0 && strip_fills(min_chunk_ctas, sms));
  const int zchunk = use_strip ? strip_zchunk(total_strips, nelz_max, sms, 0) : 0;
  int tex = e->cfg.tile_ex, tez = e->cfg.tile_ez;
  if (!use_strip && tex == 0) auto_tile(run_sv.data(), (int)run_sv.size(), sms, 256, &tex, &tez);
  // ---- descriptors and CTA maps of the running set, grouped by order
  std::vector<EngineJob*> order(e->running);
  std::stable_sort(order.begin(), order.end(),
                   [](EngineJob* x, EngineJob* y) { return x->s.plan->npol < y->s.plan->npol; });
  const int n = (int)order.size();
  e->h_solves.assign(n, SolveDev{});
  e->h_cta.clear();
  if (use_strip && n > e->tmaps_cap) {
    cudaFree(e->d_tmaps);
    e->d_tmaps = nullptr;
    e->tmaps_cap = 0;
    const int cap = std::max(n, e->cfg.max_solves);
    CUDA_TRY(cudaMalloc((void**)&e->d_tmaps, sizeof(CUtensorMap) * cap));
    e->tmaps_cap = cap;
  }
  if (use_strip) e->h_tmaps.resize(n);
  struct Group { int N; long long cta0, ncta; bool adj, stc; int first; };
  std::vector<Group> groups;
  for (int oi = 0; oi < n; ++oi) {
    EngineJob* j = order[oi];
    const sem_plan_s* p = j->s.plan;
    sem_plan_s::Lists L;
    int ntx, ntz, ntiles, rc;
    if (use_strip) {
      ntx = strips_of(p, &ntz);
      ntiles = ntx * ((p->nelz + zchunk - 1) / zchunk);
      rc = get_strip_lists(p, ntz, &L);
    } else {
      ntiles = tiles_of(p, tex, tez, &ntx, &ntz);
      rc = get_lists(p, tex, tez, &L);
    }
    if (rc) return rc;
    if (groups.empty() || groups.back().N != p->npol)
      groups.push_back(Group{p->npol, (long long)e->h_cta.size(), 0, false, false, oi});
    Group& G = groups.back();
    G.adj |= (j->s.flags & SEM_F_ADJOINT) != 0;
    G.stc |= p->bnd_n > 0;
    char* a = e->arena + j->off;
    SolveDev& d = e->h_solves[oi];
    d.nelx = p->nelx; d.nelz = p->nelz; d.nxg = p->nxg; d.nzg = p->nzg; d.pitch = p->pitch;
    d.tiles_x = ntx; d.tiles_z = ntz;
    d.zchunk = use_strip ? zchunk : p->nelz;
    d.tile_base = (int)(e->h_cta.size() - G.cta0);
    d.nt = p->nt; d.k = j->k; d.nseg = j->nseg; d.flags = j->s.flags;
    d.start_tick = (int)j->start;
    d.it0 = j->s.it0; d.it1 = j->s.it1; d.decim = j->s.decim;
    d.src_gx = p->src_gx; d.src_gz = p->src_gz; d.nrec = p->nrec;
    d.fstride = p->fstride;
    const bool adj = j->s.flags & SEM_F_ADJOINT;
    d.c2 = (const float*)(a + j->ws.c2);
    d.W = (float*)(a + j->ws.W);
    d.V = (float*)(a + j->ws.V);
    d.ckpt = adj ? (float*)(a + j->ws.ckpt) : nullptr;
    d.ring = adj ? (float*)(a + j->ws.ring) : nullptr;
    d.L = adj ? (float*)(a + j->ws.L) : nullptr;
    d.Mu = adj ? (float*)(a + j->ws.Mu) : nullptr;
    d.grad = adj ? (float*)(a + j->ws.grad) : nullptr;
    d.grad64 = adj ? (double*)(a + j->ws.grad64) : nullptr;
    d.D = p->D; d.beta = p->beta; d.tx = p->tx; d.tz = p->tz; d.src_term = p->src_term;
    d.rec_base = p->rec_base; d.rec_w = p->rec_w;
    d.rec_tile_off = L.rec_off; d.rec_tile_ids = L.rec_ids;
    d.inj_tile_off = L.inj_off; d.inj_tile_ids = L.inj_ids;
    d.rec_out = j->s.rec_out; d.yobs = j->s.y_obs;
    d.misfit = (double*)(a + j->ws.misfit);
    d.rmax = d.misfit + p->nrec;
    d.adj_scale = d.misfit + 2 * p->nrec;
    d.status = (int*)(a + j->ws.status);
    d.ws = (const float*)a;
    d.tmap = nullptr;
    d.bnd_n = p->bnd_n; d.bnd_pitch = bnd_pitch_of(p);
    d.bnd_coef = p->bnd_n ? (const float*)(a + j->ws.bnd_coef) : nullptr;
    d.bnd_hist = j->ws.bnd_hist >= 0 ? (float*)(a + j->ws.bnd_hist) : nullptr;
    if (use_strip) {
      if (!j->has_tmap) {
        rc = encode_band_map(&j->tmap, a, p, field_slots(j->ws, p, adj));
        if (rc) return rc;
        j->has_tmap = true;
      }
      e->h_tmaps[oi] = j->tmap;
      d.tmap = e->d_tmaps + oi;
    }
    for (int c = 0; c < ntiles; ++c) e->h_cta.push_back(oi - G.first);
    G.ncta += ntiles;
  }
  if (n > e->solves_cap) {
    cudaFree(e->d_solves);
    e->d_solves = nullptr;
    CUDA_TRY(cudaMalloc((void**)&e->d_solves, sizeof(SolveDev) * std::max(n, e->cfg.max_solves)));
    e->solves_cap = std::max(n, e->cfg.max_solves);
  }
  if ((long long)e->h_cta.size() > e->cta_cap) {
    cudaFree(e->d_cta);
    e->d_cta = nullptr;
    const long long cap = std::max<long long>((long long)e->h_cta.size() * 2, 1024);
    CUDA_TRY(cudaMalloc((void**)&e->d_cta, sizeof(int) * cap));
    e->cta_cap = cap;
  }
  CUDA_TRY(cudaMemcpyAsync(e->d_solves, e->h_solves.data(), sizeof(SolveDev) * n,
                           cudaMemcpyHostToDevice, stream));
  if (use_strip)
    CUDA_TRY(cudaMemcpyAsync(e->d_tmaps, e->h_tmaps.data(), sizeof(CUtensorMap) * n,
                             cudaMemcpyHostToDevice, stream));
  CUDA_TRY(cudaMemcpyAsync(e->d_cta, e->h_cta.data(), sizeof(int) * e->h_cta.size(),
                           cudaMemcpyHostToDevice, stream));
  // ---- ticks: the tick number is passed; launches chain by programmatic dependent launch
  for (int c = 0; c < e->cfg.ticks_per_step; ++c) {
    for (auto& G : groups) {
      KernelFn fn = use_strip ? strip_kernel_for(G.N) : kernel_for(G.N);
      if (!fn) return fail(SEM_ERR_UNSUPPORTED, "polynomial order");
      const size_t smem = (size_t)(use_strip ? strip_smem_floats(G.N, G.adj) + (G.stc ? kStripBndFloats : 0)
                                             : smem_floats(G.N, tex, tez, G.adj)) * sizeof(float);
      if (smem > 227 * 1024) return fail(SEM_ERR_ARG, "tile too large for shared memory");
      if (c == 0)
        CUDA_TRY(raise_smem_limit((const void*)fn, smem));
      cudaLaunchConfig_t lc = {};
      lc.gridDim = dim3((unsigned)G.ncta);
      lc.blockDim = dim3(use_strip ? strip_threads(G.N) : 256);
      lc.dynamicSmemBytes = smem;
      lc.stream = stream;
      cudaLaunchAttribute at[1];
      at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
      at[0].val.programmaticStreamSerializationAllowed = SEM_PDL ? 1 : 0;
      lc.attrs = at;
      lc.numAttrs = 1;
      const int* no_counter = nullptr;
      CUDA_TRY(cudaLaunchKernelEx(&lc, fn, (const SolveDev*)(e->d_solves + G.first),
                                  (const int*)(e->d_cta + G.cta0), no_counter, tex, tez,
                                  (int)(e->tick + c)));
      e->launches++;
    }
  }
  e->tick += e->cfg.ticks_per_step;
  CUDA_TRY(cudaGetLastError());
  return SEM_OK;
}

}  // extern "C"
