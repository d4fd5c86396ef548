// sem_velocity.cu — nodal velocity from a closed cubic B-spline interface on sm_100a.
//
// Device restatement of MUN's velocity builders
// (Bspline_Coupling/SEM/sem_waveform/velocity.py:37-202,
//  CO2_plume/layered_model/inversion/sem_waveform/velocity.py:38-267,
//  CO2_plume/one_stage/single_cubic/sem_waveform/velocity.py:54-332):
//   1. closest curve parameter: nearest of the curve samples C(u0_s), then
//      `newton_steps` Newton steps on phi(u) = |C(u) - x|^2/2 with phi'' floored at
//      1e-14 and u clipped to the valid interval;
//   2. distance to C(u*), sign from an even-odd crossing test against the sample
//      polygon (negative inside), outward normal sign * (x - C(u*)) / |x - C(u*)|;
//   3. v = v_bg + (v_in - v_bg) * sigmoid(-sd/tau) (sd/tau clipped to +-50), or the
//      hard "replace" blend.
// One thread per node, float64 throughout; the curve samples and polygon sit in shared
// memory.  Knots/coefficients describe either closure convention (clamped or periodic).

#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
#include <mutex>
#include <string>

#include "../../include/mun_sem.h"

namespace {

thread_local std::string g_verr;

// the kernel's dynamic shared-memory limit is shared by all host threads; only raise it,
// so that a concurrent call with fewer curve samples cannot lower it under a larger launch
cudaError_t raise_smem_limit(const void* fn, size_t smem) {
  static std::mutex mu;
  static std::map<int, size_t> cur;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(mu);
  size_t& c = cur[dev];
  if (smem <= c) return cudaSuccess;
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) c = smem;
  return e;
}

constexpr int kMaxCoef = 64;
constexpr int kMaxSamples = 4096;

struct CurveDev {
  int ncoef;
  double knots[kMaxCoef + 4];
  double cx[kMaxCoef], cz[kMaxCoef];    // curve coefficients
  double c1x[kMaxCoef], c1z[kMaxCoef];  // first-derivative coefficients (degree 2)
  double c2x[kMaxCoef], c2z[kMaxCoef];  // second-derivative coefficients (degree 1)
  double lo, hi;
};

// explicit rounding: no contraction into FMAs, so the device follows the host's
// arithmetic step by step (the closest-point Newton iteration is sensitive to rounding
// near the curve's medial axis)
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }

// value, first and second derivative at u: de Boor basis triangle of degrees 0..3 at the
// span t[i] <= u < t[i+1] (clamped to the last valid span), contracted with the curve
// coefficients and the differenced derivative coefficients
__device__ void curve_eval(const CurveDev& c, double u, double* C, double* C1, double* C2) {
  const int k = 3;
  int i = k;
  for (int j = k; j < c.ncoef; ++j)
    if (c.knots[j] <= u) i = j;
  double N[4][4];  // N[deg][r] = N_{i-deg+r, deg}(u)
  N[0][0] = 1.0;
  double left[4], right[4];
  for (int j = 1; j <= k; ++j) {
    left[j] = sub(u, c.knots[i + 1 - j]);
    right[j] = sub(c.knots[i + j], u);
    double saved = 0.0;
    for (int r = 0; r < j; ++r) {
      const double denom = add(right[r + 1], left[j - r]);
      const double temp = (denom != 0.0) ? __ddiv_rn(N[j - 1][r], denom) : 0.0;
      N[j][r] = add(saved, mul(right[r + 1], temp));
      saved = mul(left[j - r], temp);
    }
    N[j][j] = saved;
  }
  double x0 = 0, z0 = 0, x1 = 0, z1 = 0, x2 = 0, z2 = 0;
  for (int j = 0; j <= 3; ++j) {
    x0 = add(x0, mul(N[3][j], c.cx[i - 3 + j]));
    z0 = add(z0, mul(N[3][j], c.cz[i - 3 + j]));
  }
  for (int j = 0; j <= 2; ++j) {
    x1 = add(x1, mul(N[2][j], c.c1x[i - 2 + j]));
    z1 = add(z1, mul(N[2][j], c.c1z[i - 2 + j]));
  }
  for (int j = 0; j <= 1; ++j) {
    x2 = add(x2, mul(N[1][j], c.c2x[i - 1 + j]));
    z2 = add(z2, mul(N[1][j], c.c2z[i - 1 + j]));
  }
  C[0] = x0; C[1] = z0; C1[0] = x1; C1[1] = z1; C2[0] = x2; C2[1] = z2;
}

__global__ void velocity_kernel(CurveDev curve, const double* __restrict__ u0,
                                const double* __restrict__ samples, int ns, int newton_steps,
                                const double* __restrict__ coords, int n,
                                const double* __restrict__ v_bg, double v_out, double v_in,
                                double tau, int blend_replace, double* __restrict__ vel,
                                double* __restrict__ sd_out, double* __restrict__ u_out,
                                double* __restrict__ n_out) {
  extern __shared__ double sm[];
  double* sx = sm;
  double* sz = sm + ns;
  for (int i = threadIdx.x; i < ns; i += blockDim.x) { sx[i] = samples[2 * i]; sz[i] = samples[2 * i + 1]; }
  __syncthreads();
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const double X = coords[2 * p], Z = coords[2 * p + 1];
  // nearest sample (first minimum, like argmin)
  int best = 0;
  double bd = __dadd_rn(__dmul_rn(X - sx[0], X - sx[0]), __dmul_rn(Z - sz[0], Z - sz[0]));
  for (int s = 1; s < ns; ++s) {
    const double dx = X - sx[s], dz = Z - sz[s];
    const double d2 = __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dz, dz));
    if (d2 < bd) { bd = d2; best = s; }
  }
  double u = u0[best];
  double C[2], C1[2], C2[2];
  for (int it = 0; it < newton_steps; ++it) {
    curve_eval(curve, u, C, C1, C2);
    const double rx = sub(C[0], X), rz = sub(C[1], Z);
    const double f1 = add(mul(rx, C1[0]), mul(rz, C1[1]));
    double f2 = add(add(mul(C1[0], C1[0]), mul(C1[1], C1[1])), add(mul(rx, C2[0]), mul(rz, C2[1])));
    if (fabs(f2) < 1e-14) f2 = 1e-14;
    u = fmin(fmax(sub(u, __ddiv_rn(f1, f2)), curve.lo), curve.hi);
  }
  curve_eval(curve, u, C, C1, C2);
  const double rvx = sub(X, C[0]), rvz = sub(Z, C[1]);
  const double dist = __dsqrt_rn(add(mul(rvx, rvx), mul(rvz, rvz)));
  // even-odd crossing test against the closed sample polygon
  bool inside = false;
  for (int s = 0; s < ns; ++s) {
    const int t = (s + 1 == ns) ? 0 : s + 1;
    const double ay = sz[s], by = sz[t];
    if (ay == by) continue;
    if ((ay > Z) != (by > Z)) {
      const double xc = add(sx[s], __ddiv_rn(mul(sub(Z, ay), sub(sx[t], sx[s])), sub(by, ay)));
      if (X < xc) inside = !inside;
    }
  }
  const double sign = inside ? -1.0 : 1.0;
  const double sd = sign * dist;
  const double bg = v_bg ? v_bg[p] : v_out;
  double v;
  if (blend_replace) {
    v = (sd < 0.0) ? v_in : bg;
  } else {
    const double ts = fmax(tau, 1e-12);
    const double x = fmin(fmax(sd / ts, -50.0), 50.0);
    const double sig = 1.0 / (1.0 + exp(x));
    v = bg + (v_in - bg) * sig;
  }
  vel[p] = v;
  if (sd_out) sd_out[p] = sd;
  if (u_out) u_out[p] = u;
  if (n_out) {
    n_out[2 * p] = mul(sign, __ddiv_rn(rvx, add(dist, 1e-15)));
    n_out[2 * p + 1] = mul(sign, __ddiv_rn(rvz, add(dist, 1e-15)));
  }
}

// Control-point projection of dL/dv for a batch of samples (row s of every (S, P) input):
//   dv_p = (v_in - bg_p) sig_p (1 - sig_p) (-1/tau),  sig_p = 1 / (1 + exp(clip(sd_p/tau, +-50)))
//   mask: |dv_p| > 1e-8 * (floor_one ? max(1, |v_in - bg_p|) : |v_in - bg_p|)
//   out[s][j]     = sum_p mask w_p B_j(u_p) n_p,x,   out[s][K + j] = ... n_p,z,  w_p = dL_p dv_p
// B_j is the cubic basis at the closest-point parameter (periodic curves: the gridded
// package's mapping t = lo + mod(u, 1) (hi - lo)), with the duplicated closing controls
// folded back onto the points they copy.  One block per (sample, control point); each
// thread sums a fixed node subset, then a fixed-order tree: deterministic.
__global__ void project_kernel(CurveDev curve, int K, int periodic, int P, const double* __restrict__ dL,
                               const double* __restrict__ sd, const double* __restrict__ us,
                               const double* __restrict__ nrm, const double* __restrict__ bg,
                               double bg_const, double v_in, double tau, int floor_one,
                               double* __restrict__ out) {
  const int j = blockIdx.x, smp = blockIdx.y;
  const long long row = (long long)smp * P;
  const double ts = fmax(tau, 1e-12);
  double ax = 0.0, az = 0.0;
  for (int p = threadIdx.x; p < P; p += blockDim.x) {
    const double b = bg ? bg[p] : bg_const;
    const double delta = v_in - b;
    const double x = fmin(fmax(sd[row + p] / ts, -50.0), 50.0);
    const double sig = 1.0 / (1.0 + exp(x));
    const double dv = delta * sig * (1.0 - sig) * (-1.0 / ts);
    const double lim = 1e-8 * (floor_one ? fmax(1.0, fabs(delta)) : fabs(delta));
    if (!(fabs(dv) > lim)) continue;
    double u = us[row + p];
    if (periodic) {
      const double fr = u - floor(u);  // mod(u, 1)
      u = fmin(fmax(curve.lo + fr * (curve.hi - curve.lo), curve.lo), nextafter(curve.hi, curve.lo));
    }
    // span i: t[i] <= u < t[i+1], clamped to the last valid span
    int i = 3;
    for (int q = 3; q < curve.ncoef; ++q)
      if (curve.knots[q] <= u) i = q;
    double Nb[4][4];
    Nb[0][0] = 1.0;
    double left[4], right[4];
    for (int d = 1; d <= 3; ++d) {
      left[d] = u - curve.knots[i + 1 - d];
      right[d] = curve.knots[i + d] - u;
      double saved = 0.0;
      for (int r = 0; r < d; ++r) {
        const double den = right[r + 1] + left[d - r];
        const double tmp = (den != 0.0) ? Nb[d - 1][r] / den : 0.0;
        Nb[d][r] = saved + right[r + 1] * tmp;
        saved = left[d - r] * tmp;
      }
      Nb[d][d] = saved;
    }
    double bj = 0.0;
    for (int r = 0; r < 4; ++r) {
      const int c = i - 3 + r;
      const int f = (c < K) ? c : (periodic ? c - K : 0);
      if (f == j) bj += Nb[3][r];
    }
    if (bj == 0.0) continue;
    const double w = dL[row + p] * dv;
    ax += w * bj * nrm[2 * (row + p)];
    az += w * bj * nrm[2 * (row + p) + 1];
  }
  __shared__ double sx[256], sz[256];
  sx[threadIdx.x] = ax;
  sz[threadIdx.x] = az;
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) {
      sx[threadIdx.x] += sx[threadIdx.x + h];
      sz[threadIdx.x] += sz[threadIdx.x + h];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[(long long)smp * 2 * K + j] = sx[0];
    out[(long long)smp * 2 * K + K + j] = sz[0];
  }
}

}  // namespace

extern "C" {

int sem_project_from_curve(const double* knots, int32_t ncoef, int32_t K, int32_t periodic,
                           int32_t nsamples, int32_t npoints, const double* dL_dv, const double* sd,
                           const double* ustar, const double* normal, const double* v_background,
                           double v_background_const, double v_inside, double tau, int32_t floor_one,
                           double* grad_out, void* stream) {
  if (!knots || !dL_dv || !sd || !ustar || !normal || !grad_out) {
    g_verr = "null argument";
    return SEM_ERR_ARG;
  }
  if (ncoef < 4 || ncoef > kMaxCoef || K < 1 || K > ncoef || nsamples < 0 || npoints < 0 ||
      nsamples > 65535) {
    g_verr = "bad curve size, control-point count or batch size";
    return SEM_ERR_ARG;
  }
  if (nsamples == 0) return SEM_OK;
  CurveDev cd{};
  cd.ncoef = ncoef;
  for (int i = 0; i < ncoef + 4; ++i) cd.knots[i] = knots[i];
  cd.lo = knots[3];
  cd.hi = knots[ncoef];
  project_kernel<<<dim3((unsigned)K, (unsigned)nsamples), 256, 0, (cudaStream_t)stream>>>(
      cd, K, periodic, npoints, dL_dv, sd, ustar, normal, v_background, v_background_const, v_inside,
      tau, floor_one, grad_out);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) { g_verr = cudaGetErrorString(e); return SEM_ERR_CUDA; }
  return SEM_OK;
}

const char* sem_velocity_last_error(void) { return g_verr.c_str(); }

int sem_velocity_from_curve(const sem_curve_t* c, int32_t npoints, const double* coords,
                            const double* v_background, double v_outside, double* velocity_out,
                            double* sd_out, double* ustar_out, double* normal_out, void* stream) {
  if (!c || !coords || !velocity_out || !c->knots || !c->coef || !c->u0 || !c->samples) {
    g_verr = "null argument";
    return SEM_ERR_ARG;
  }
  if (c->ncoef < 4 || c->ncoef > kMaxCoef || c->nsamples < 3 || c->nsamples > kMaxSamples ||
      c->newton_steps < 0 || npoints < 0) {
    g_verr = "curve has too many control points or samples";
    return SEM_ERR_ARG;
  }
  CurveDev cd{};
  cd.ncoef = c->ncoef;
  for (int i = 0; i < c->ncoef + 4; ++i) cd.knots[i] = c->knots[i];
  for (int i = 0; i < c->ncoef; ++i) { cd.cx[i] = c->coef[2 * i]; cd.cz[i] = c->coef[2 * i + 1]; }
  // derivative coefficients: d/du sum c_j N_{j,k} = sum k (c_j - c_{j-1}) / (t_{j+k} - t_j) N_{j,k-1}
  for (int i = 0; i < c->ncoef; ++i) {
    const double den = cd.knots[i + 3] - cd.knots[i];
    cd.c1x[i] = (i >= 1 && den > 0) ? 3.0 * (cd.cx[i] - cd.cx[i - 1]) / den : 0.0;
    cd.c1z[i] = (i >= 1 && den > 0) ? 3.0 * (cd.cz[i] - cd.cz[i - 1]) / den : 0.0;
  }
  for (int i = 0; i < c->ncoef; ++i) {
    const double den = cd.knots[i + 2] - cd.knots[i];
    cd.c2x[i] = (i >= 1 && den > 0) ? 2.0 * (cd.c1x[i] - cd.c1x[i - 1]) / den : 0.0;
    cd.c2z[i] = (i >= 1 && den > 0) ? 2.0 * (cd.c1z[i] - cd.c1z[i - 1]) / den : 0.0;
  }
  cd.lo = c->u_lo;
  cd.hi = c->u_hi;
  if (npoints == 0) return SEM_OK;
  const int threads = 128;
  const size_t smem = (size_t)2 * c->nsamples * sizeof(double);
  cudaError_t e = raise_smem_limit((const void*)velocity_kernel, smem);
  if (e != cudaSuccess) { g_verr = cudaGetErrorString(e); return SEM_ERR_CUDA; }
  velocity_kernel<<<(npoints + threads - 1) / threads, threads, smem, (cudaStream_t)stream>>>(
      cd, c->u0, c->samples, c->nsamples, c->newton_steps, coords, npoints, v_background,
      v_outside, c->v_inside, c->tau, c->blend_replace, velocity_out, sd_out, ustar_out, normal_out);
  e = cudaGetLastError();
  if (e != cudaSuccess) { g_verr = cudaGetErrorString(e); return SEM_ERR_CUDA; }
  return SEM_OK;
}

}  // extern "C"
