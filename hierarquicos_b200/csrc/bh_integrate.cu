// Time integration on the device: the kick and drift updates of the
// reference's integrators, and the conserved-quantity diagnostics.
//
// State is momentum form, FP64, structure of arrays over a batch of systems
// stored back to back (system s owns bodies [off[s], off[s+1])).  Forces come
// in the layout the walk writes: one (n_s, 3) Fortran block per system at
// 3 off[s].
//
// The updates repeat the reference's operation order, without contraction:
//   velocity Verlet (parareal/parareal.f90:55-63, integration.f90:152-168)
//     p_half = p + (0.5 dt) f ;  q = q + (dt p_half) / m ;  f = F(q) ;
//     p = p_half + (0.5 dt) f
//   symplectic Euler, the coarse propagator (parareal/parareal.f90:20-35)
//     p = p + dt f ;  q = q + (dt p) / m
// A step boundary of Verlet (closing half kick, next opening half kick, drift)
// is one launch: p = (p + k1 f) + k2 f, then the drift.
#include "bh_internal.cuh"

namespace bh {
namespace {

__device__ __forceinline__ int system_of(const int64_t *__restrict__ off, int nsys, int64_t g) {
  int a = 0, b = nsys;  // largest s with off[s] <= g
  while (b - a > 1) {
    const int mid = (a + b) >> 1;
    if (off[mid] <= g) a = mid; else b = mid;
  }
  return a;
}

__global__ void __launch_bounds__(256)
kick_drift_kernel(const double *__restrict__ m, const double *__restrict__ f,
                  double *__restrict__ x, double *__restrict__ y, double *__restrict__ z,
                  double *__restrict__ px, double *__restrict__ py, double *__restrict__ pz,
                  const int64_t *__restrict__ off, int nsys, int64_t n, double k1_all,
                  double k2_all, double dt_all, const double *__restrict__ coef) {
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < n;
       g += (int64_t)gridDim.x * blockDim.x) {
    double p0 = px[g], p1 = py[g], p2 = pz[g];
    const int s = system_of(off, nsys, g);
    // coefficients of the whole batch, or of each system (coef: 3 per system)
    const double k1 = coef ? coef[3 * s] : k1_all;
    const double k2 = coef ? coef[3 * s + 1] : k2_all;
    const double dt = coef ? coef[3 * s + 2] : dt_all;
    if (k1 != 0.0 || k2 != 0.0) {
      const int64_t ns = off[s + 1] - off[s], i = g - off[s];
      const double *fs = f + 3 * off[s];
      const double f0 = fs[i], f1 = fs[ns + i], f2 = fs[2 * ns + i];
      if (k1 != 0.0) {
        p0 = __dadd_rn(p0, __dmul_rn(k1, f0));
        p1 = __dadd_rn(p1, __dmul_rn(k1, f1));
        p2 = __dadd_rn(p2, __dmul_rn(k1, f2));
      }
      if (k2 != 0.0) {
        p0 = __dadd_rn(p0, __dmul_rn(k2, f0));
        p1 = __dadd_rn(p1, __dmul_rn(k2, f1));
        p2 = __dadd_rn(p2, __dmul_rn(k2, f2));
      }
      px[g] = p0; py[g] = p1; pz[g] = p2;
    }
    if (dt != 0.0) {
      const double mg = m[g];
      x[g] = __dadd_rn(x[g], __ddiv_rn(__dmul_rn(dt, p0), mg));
      y[g] = __dadd_rn(y[g], __ddiv_rn(__dmul_rn(dt, p1), mg));
      z[g] = __dadd_rn(z[g], __ddiv_rn(__dmul_rn(dt, p2), mg));
    }
  }
}

// Per-body sums for the diagnostics (parareal/api3d.f90:108-153): kinetic
// energy p.p / (2 m), half the pair potential -G m_a m_b / sqrt(r^2 + eps^2)
// over the other bodies of the system, linear momentum p and angular momentum
// q x p.  One block per 128 targets; sources of the target's system staged
// through shared memory.  A block's targets may span systems: each target
// only sums over its own.
constexpr int kDiagThreads = 128;

__global__ void __launch_bounds__(kDiagThreads)
diag_body_kernel(const double *__restrict__ m, const double *__restrict__ x,
                 const double *__restrict__ y, const double *__restrict__ z,
                 const double *__restrict__ px, const double *__restrict__ py,
                 const double *__restrict__ pz, const int64_t *__restrict__ off, int nsys,
                 int64_t n, double G, double eps2, double *__restrict__ per_body) {
  __shared__ double4 src[kDiagThreads];
  const int64_t g0 = (int64_t)blockIdx.x * kDiagThreads;
  const int64_t g = g0 + threadIdx.x;
  const bool valid = g < n;
  const int64_t gl = valid ? g : n - 1;
  const int s = system_of(off, nsys, gl);
  // the systems this block touches: [s_first, s_last]
  const int s_first = system_of(off, nsys, g0);
  const int s_last = system_of(off, nsys, bh_min64(g0 + kDiagThreads, n) - 1);
  const double qa0 = x[gl], qa1 = y[gl], qa2 = z[gl], ma = m[gl];
  double pot = 0.0;
  for (int t = s_first; t <= s_last; ++t) {
    for (int64_t base = off[t]; base < off[t + 1]; base += kDiagThreads) {
      __syncthreads();
      const int64_t b = base + threadIdx.x;
      src[threadIdx.x] = b < off[t + 1] ? make_double4(x[b], y[b], z[b], m[b])
                                        : make_double4(0.0, 0.0, 0.0, 0.0);
      __syncthreads();
      if (t != s) continue;
      const int cnt = (int)bh_min64(kDiagThreads, off[t + 1] - base);
      for (int j = 0; j < cnt; ++j) {
        if (base + j == gl) continue;
        const double4 q = src[j];
        const double dx = q.x - qa0, dy = q.y - qa1, dz = q.z - qa2;
        const double r = sqrt(dx * dx + dy * dy + dz * dz + eps2);
        pot -= G * ma * q.w / r;
      }
    }
  }
  if (!valid) return;
  const double p0 = px[g], p1 = py[g], p2 = pz[g];
  double *o = per_body + 8 * g;
  o[0] = 0.5 * (p0 * p0 + p1 * p1 + p2 * p2) / ma;
  o[1] = 0.5 * pot;
  o[2] = p0; o[3] = p1; o[4] = p2;
  o[5] = qa1 * p2 - p1 * qa2;
  o[6] = -qa0 * p2 + p0 * qa2;
  o[7] = qa0 * p1 - p0 * qa1;
}

// Fixed-order reduction of the per-body sums, one block per system.
__global__ void __launch_bounds__(256)
diag_reduce_kernel(const double *__restrict__ per_body, const int64_t *__restrict__ off,
                   double *__restrict__ out) {
  __shared__ double red[8][256];
  const int s = blockIdx.x;
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int64_t g = off[s] + threadIdx.x; g < off[s + 1]; g += blockDim.x)
    for (int k = 0; k < 8; ++k) acc[k] += per_body[8 * g + k];
  for (int k = 0; k < 8; ++k) red[k][threadIdx.x] = acc[k];
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
      for (int k = 0; k < 8; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x < 8) {
    const double v = red[threadIdx.x][0];
    // out: E = kinetic + potential, then kinetic, potential, P(3), J(3)
    double *o = out + 9 * s;
    if (threadIdx.x == 0) o[1] = v;
    else if (threadIdx.x == 1) o[2] = v;
    else o[threadIdx.x + 1] = v;
  }
  __syncthreads();
  if (threadIdx.x == 0) out[9 * s] = red[0][0] + red[1][0];
}

}  // namespace

void launch_kick_drift(const double *m, const double *f, double *x, double *y, double *z,
                       double *px, double *py, double *pz, const int64_t *off, int nsys, int64_t n,
                       double k1, double k2, double dt, const double *coef, cudaStream_t s) {
  kick_drift_kernel<<<grid_for(n, 256, 148 * 16), 256, 0, s>>>(m, f, x, y, z, px, py, pz, off,
                                                               nsys, n, k1, k2, dt, coef);
}

void launch_diagnostics(const double *m, const double *x, const double *y, const double *z,
                        const double *px, const double *py, const double *pz, const int64_t *off,
                        int nsys, int64_t n, double G, double eps, double *scratch, double *out,
                        cudaStream_t s) {
  const int blocks = (int)((n + kDiagThreads - 1) / kDiagThreads);
  diag_body_kernel<<<blocks, kDiagThreads, 0, s>>>(m, x, y, z, px, py, pz, off, nsys, n, G,
                                                   eps * eps, scratch);
  diag_reduce_kernel<<<nsys, 256, 0, s>>>(scratch, off, out);
}

}  // namespace bh

extern "C" {

int bh_kick_drift(const double *d_m, const double *d_f, double *d_x, double *d_y, double *d_z,
                  double *d_px, double *d_py, double *d_pz, const int64_t *d_offsets, int nsys,
                  int64_t n, double kick1, double kick2, double drift, void *stream) {
  if (n < 1 || nsys < 1 || !d_offsets || !d_m || !d_x || !d_y || !d_z || !d_px || !d_py || !d_pz)
    return bh_report_error(BH_ERR_INVALID, "bh_kick_drift: bad arguments");
  if ((kick1 != 0.0 || kick2 != 0.0) && !d_f)
    return bh_report_error(BH_ERR_INVALID, "bh_kick_drift: a kick needs forces");
  bh::launch_kick_drift(d_m, d_f, d_x, d_y, d_z, d_px, d_py, d_pz, d_offsets, nsys, n, kick1,
                        kick2, drift, nullptr, (cudaStream_t)stream);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return bh_report_error(BH_ERR_CUDA, cudaGetErrorString(e));
  return BH_OK;
}

int bh_kick_drift_systems(const double *d_m, const double *d_f, double *d_x, double *d_y,
                          double *d_z, double *d_px, double *d_py, double *d_pz,
                          const int64_t *d_offsets, int nsys, int64_t n, const double *d_coef,
                          void *stream) {
  if (n < 1 || nsys < 1 || !d_offsets || !d_m || !d_x || !d_y || !d_z || !d_px || !d_py ||
      !d_pz || !d_coef || !d_f)
    return bh_report_error(BH_ERR_INVALID, "bh_kick_drift_systems: bad arguments");
  bh::launch_kick_drift(d_m, d_f, d_x, d_y, d_z, d_px, d_py, d_pz, d_offsets, nsys, n, 0.0, 0.0,
                        0.0, d_coef, (cudaStream_t)stream);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return bh_report_error(BH_ERR_CUDA, cudaGetErrorString(e));
  return BH_OK;
}

int bh_diagnostics(const double *d_m, const double *d_x, const double *d_y, const double *d_z,
                   const double *d_px, const double *d_py, const double *d_pz,
                   const int64_t *d_offsets, int nsys, int64_t n, double G, double eps,
                   double *d_scratch, double *d_out, void *stream) {
  if (n < 1 || nsys < 1 || !d_offsets || !d_m || !d_x || !d_y || !d_z || !d_px || !d_py ||
      !d_pz || !d_scratch || !d_out)
    return bh_report_error(BH_ERR_INVALID, "bh_diagnostics: bad arguments");
  bh::launch_diagnostics(d_m, d_x, d_y, d_z, d_px, d_py, d_pz, d_offsets, nsys, n, G, eps,
                         d_scratch, d_out, (cudaStream_t)stream);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return bh_report_error(BH_ERR_CUDA, cudaGetErrorString(e));
  return BH_OK;
}

}  // extern "C"
