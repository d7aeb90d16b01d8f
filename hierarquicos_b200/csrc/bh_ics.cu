// Initial conditions generated on the device (seeded, counter-based).
//
// Mirrors initial_values/initial_values.f90:51-381 and the profile modules
// (plummer.f90, hernquist.f90, homogeneous.f90): radius by inverting the
// cumulative mass P(r) (rejected above size_qs when size_qs >= 0), isotropic
// direction (phi = 2 pi X, cos theta = 2 X - 1), speed by von Neumann sampling
// of q = v / v_esc from q^2 f(E) (Plummer, Hernquist) or uniform in
// [-size_ps, size_ps] (uniform sphere, homogeneous), isotropic velocity
// direction, momenta p = m v, then the total momentum and the centre of mass
// moved to zero.
//
// Random numbers: every body draws from its own counter-based stream, so the
// result does not depend on the launch shape.  A draw is the SplitMix64
// finaliser (Steele, Lea and Flood, OOPSLA 2014) of (seed, stream, body,
// counter), mapped to [0, 1) with 53 bits.  The streams differ from the host
// generator's (NumPy PCG64); the distributions are the same.
#include <math.h>

#include "bh_internal.cuh"

namespace bh {
namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr int kMaxTries = 100000;

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

struct Stream {
  uint64_t key;
  uint64_t ctr;
  __device__ Stream(uint64_t seed, uint64_t stream, uint64_t body)
      : key(mix64(mix64(seed + 0x9e3779b97f4a7c15ull * (stream + 1)) ^ body)), ctr(0) {}
  __device__ __forceinline__ double uniform() {
    const uint64_t r = mix64(key + 0x9e3779b97f4a7c15ull * (++ctr));
    return (double)(r >> 11) * 0x1.0p-53;
  }
};

enum Profile : int { kUniform = 0, kUniformSphere = 1, kPlummer = 2, kHomogeneous = 3, kHernquist = 4 };

__device__ double inverse_P(int prof, double x, double par) {
  switch (prof) {
    case kPlummer:  // plummer.f90:53-62
      return pow(x, 1.0 / 3.0) * par / sqrt(1.0 - pow(x, 2.0 / 3.0));
    case kHomogeneous:  // homogeneous.f90:48-61
      return par * pow(x, 1.0 / 3.0);
    case kHernquist:  // hernquist.f90:158-171
      return par * sqrt(x) / (1.0 - sqrt(x));
  }
  return 0.0;
}

__device__ double hernquist_edf_norm(double r, double x, double G, double a) {
  // hernquist.f90:200-212
  const double E = sqrt(G / (a + r) * (1.0 - x * x));
  double edf = 1.0 / (8.0 * sqrt(2.0) * a * kPi * kPi * kPi);
  edf = edf / pow(sqrt(1.0 - E), 5.0);
  edf = edf * 3.0 * asin(sqrt(E));
  return edf + edf * sqrt(E * (1.0 - E)) * (1.0 - 2.0 * E) * (8.0 * E * E - 8.0 * E - 3.0);
}

__device__ double hernquist_maximum_pdf(double r, double G, double a) {
  // hernquist.f90:214-247: first sign change of d/dq [q^2 f] (centred
  // differences, h = 1e-3)
  const double h = 0.001;
  auto der = [&](double x) {
    return ((x + h) * (x + h) * hernquist_edf_norm(r, x + h, G, a) -
            (x - h) * (x - h) * hernquist_edf_norm(r, x - h, G, a)) / (2.0 * h);
  };
  double x = h, before = der(x);
  while (x + h < 1.0) {
    x += h;
    const double next = der(x);
    if (before * next <= 0.0) return x * x * hernquist_edf_norm(r, x, G, a);
    before = next;
  }
  return 1.0;
}

__device__ void direction(Stream &rng, int two_d, double len, double &x, double &y, double &z) {
  // initial_values.f90:355-381
  const double phi = 2.0 * kPi * rng.uniform();
  double ct = 0.0, st = 1.0;
  if (!two_d) {
    ct = 2.0 * rng.uniform() - 1.0;
    st = sqrt(1.0 - ct * ct);
  }
  x = len * st * cos(phi);
  y = len * st * sin(phi);
  z = len * ct;
}

__global__ void __launch_bounds__(256)
ics_kernel(int prof, int64_t n, double size_qs, double size_ps, int two_d, int nm, double G,
           double par, uint64_t seed, int velocities, double *__restrict__ m,
           double *__restrict__ q, double *__restrict__ p, int *__restrict__ err) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    Stream rq(seed, 0, (uint64_t)i), rv(seed, 1, (uint64_t)i), rm(seed, 2, (uint64_t)i);
    double qx, qy, qz, vx = 0.0, vy = 0.0, vz = 0.0;
    double r = 0.0;
    if (prof == kUniform) {
      qx = size_qs * (2.0 * rq.uniform() - 1.0);
      qy = size_qs * (2.0 * rq.uniform() - 1.0);
      qz = size_qs * (2.0 * rq.uniform() - 1.0);
      if (velocities) {
        vx = size_ps * (2.0 * rv.uniform() - 1.0);
        vy = size_ps * (2.0 * rv.uniform() - 1.0);
        vz = size_ps * (2.0 * rv.uniform() - 1.0);
      }
    } else {
      if (prof == kUniformSphere) {
        r = size_qs * (2.0 * rq.uniform() - 1.0);
      } else {
        int t = 0;
        for (; t < kMaxTries; ++t) {
          r = inverse_P(prof, rq.uniform(), par);
          if (!(size_qs >= 0.0 && r > size_qs)) break;
        }
        if (t == kMaxTries) atomicOr(err, 1);
      }
      direction(rq, two_d, r, qx, qy, qz);
      if (velocities) {
        double vr = 0.0;
        if (prof == kPlummer || prof == kHernquist) {
          const double pot = prof == kPlummer ? -G / sqrt(r * r + par * par) : -G / (par + r);
          const double vesc = sqrt(-2.0 * pot);
          const double mx = prof == kPlummer ? 0.0922108113291 : hernquist_maximum_pdf(r, G, par);
          int t = 0;
          double qv = 0.0;
          for (; t < kMaxTries; ++t) {
            const double y = mx * rv.uniform();
            qv = rv.uniform();
            const double pdf = prof == kPlummer ? qv * qv * pow(1.0 - qv * qv, 3.5)
                                                : qv * qv * hernquist_edf_norm(r, qv, G, par);
            if (y < pdf) break;
          }
          if (t == kMaxTries) atomicOr(err, 2);
          vr = qv * vesc;
        } else {
          vr = size_ps * (2.0 * rv.uniform() - 1.0);
        }
        direction(rv, two_d, vr, vx, vy, vz);
      }
    }
    if (two_d) { qz = 0.0; vz = 0.0; }
    q[i] = qx; q[n + i] = qy; q[2 * n + i] = qz;
    p[i] = vx; p[n + i] = vy; p[2 * n + i] = vz;  // velocities until the mass pass
    if (!nm) {
      double u = rm.uniform();
      for (int t = 0; u == 0.0 && t < 64; ++t) u = rm.uniform();
      m[i] = u;  // normalised below
    } else {
      m[i] = 1.0 / (double)n;
    }
  }
}

// Fixed-order sums over all bodies: block partials of
// (m, m x, m y, m z, p x, p y, p z, max |v|) then one block folds them.
constexpr int kSumThreads = 256;
constexpr int kSumBlocks = 296;

__global__ void __launch_bounds__(kSumThreads)
ics_partials_kernel(int64_t n, const double *__restrict__ m, const double *__restrict__ q,
                    const double *__restrict__ v, int use_mass_in_v, double *__restrict__ part) {
  __shared__ double red[8][kSumThreads];
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double mi = m[i];
    acc[0] += mi;
    acc[1] += mi * q[i];
    acc[2] += mi * q[n + i];
    acc[3] += mi * q[2 * n + i];
    const double s = use_mass_in_v ? mi : 1.0;
    acc[4] += s * v[i];
    acc[5] += s * v[n + i];
    acc[6] += s * v[2 * n + i];
    acc[7] = fmax(acc[7], fmax(fabs(v[i]), fmax(fabs(v[n + i]), fabs(v[2 * n + i]))));
  }
  for (int k = 0; k < 8; ++k) red[k][threadIdx.x] = acc[k];
  __syncthreads();
  for (int w = kSumThreads / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
      for (int k = 0; k < 8; ++k)
        red[k][threadIdx.x] = k == 7 ? fmax(red[k][threadIdx.x], red[k][threadIdx.x + w])
                                     : red[k][threadIdx.x] + red[k][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x < 8) part[8 * blockIdx.x + threadIdx.x] = red[threadIdx.x][0];
}

__global__ void ics_fold_kernel(const double *__restrict__ part, int nparts,
                                double *__restrict__ tot) {
  if (threadIdx.x >= 8) return;
  const int k = threadIdx.x;
  double a = 0.0;
  for (int b = 0; b < nparts; ++b) a = k == 7 ? fmax(a, part[8 * b + k]) : a + part[8 * b + k];
  tot[k] = a;
}

// masses normalised (random masses), velocities scaled to size_ps, momenta
// p = m v, total momentum and centre of mass removed (initial_values.f90:
// 120-173)
__global__ void __launch_bounds__(256)
ics_finish_kernel(int64_t n, int nm, double size_ps, int velocities, int two_d,
                  const double *__restrict__ tot_v, double *__restrict__ m,
                  double *__restrict__ q, double *__restrict__ p) {
  const double msum = tot_v[0];
  const double vmax = tot_v[7];
  const double vscale = (velocities && size_ps >= 0.0 && vmax > size_ps) ? size_ps / vmax : 1.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double mi = nm ? m[i] : m[i] / msum;
    m[i] = mi;
    for (int k = 0; k < 3; ++k) p[k * n + i] = p[k * n + i] * vscale * mi;
    if (two_d) p[2 * n + i] = 0.0;
  }
}

__global__ void __launch_bounds__(256)
ics_center_kernel(int64_t n, const double *__restrict__ tot, double *__restrict__ q,
                  double *__restrict__ p) {
  const double msum = tot[0];
  const double c[3] = {tot[1] / msum, tot[2] / msum, tot[3] / msum};
  const double pm[3] = {tot[4] / (double)n, tot[5] / (double)n, tot[6] / (double)n};
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    for (int k = 0; k < 3; ++k) {
      p[k * n + i] -= pm[k];
      q[k * n + i] -= c[k];
    }
}

}  // namespace
}  // namespace bh

extern "C" int bh_generate_ics(int profile, int64_t n, double size_qs, double size_ps, int two_d,
                               int nm, double G, double par, uint64_t seed, int velocities,
                               double *d_m, double *d_q, double *d_p, double *d_scratch,
                               void *stream) {
  if (profile < 0 || profile > 4) return bh_report_error(BH_ERR_INVALID, "unknown profile");
  if (n < 1 || !d_m || !d_q || !d_p || !d_scratch)
    return bh_report_error(BH_ERR_INVALID, "bh_generate_ics: bad arguments");
  if ((profile == bh::kPlummer || profile == bh::kHernquist || profile == bh::kHomogeneous) &&
      !(par > 0.0))
    return bh_report_error(BH_ERR_INVALID, "profile parameter must be > 0");
  cudaStream_t s = (cudaStream_t)stream;
  int *err = reinterpret_cast<int *>(d_scratch + 8 * bh::kSumBlocks + 16);
  cudaMemsetAsync(err, 0, sizeof(int), s);
  const int grid = bh::grid_for(n, 256, 148 * 16);
  bh::ics_kernel<<<grid, 256, 0, s>>>(profile, n, size_qs, size_ps, two_d, nm, G, par, seed,
                                      velocities, d_m, d_q, d_p, err);
  double *part = d_scratch, *tot = d_scratch + 8 * bh::kSumBlocks;
  // masses and velocity scale from the raw draws
  bh::ics_partials_kernel<<<bh::kSumBlocks, bh::kSumThreads, 0, s>>>(n, d_m, d_q, d_p, 0, part);
  bh::ics_fold_kernel<<<1, 32, 0, s>>>(part, bh::kSumBlocks, tot);
  bh::ics_finish_kernel<<<grid, 256, 0, s>>>(n, nm, size_ps, velocities, two_d, tot, d_m, d_q,
                                             d_p);
  // centre of mass and total momentum of the final masses and momenta
  bh::ics_partials_kernel<<<bh::kSumBlocks, bh::kSumThreads, 0, s>>>(n, d_m, d_q, d_p, 0, part);
  bh::ics_fold_kernel<<<1, 32, 0, s>>>(part, bh::kSumBlocks, tot);
  bh::ics_center_kernel<<<grid, 256, 0, s>>>(n, tot, d_q, d_p);
  int h_err = 0;
  cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, s);
  const cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return bh_report_error(BH_ERR_CUDA, cudaGetErrorString(e));
  if (h_err) return bh_report_error(BH_ERR_INTERNAL, "too many rejection-sampling attempts");
  return BH_OK;
}
