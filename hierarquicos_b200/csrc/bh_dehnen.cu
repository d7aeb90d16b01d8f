// Dehnen's dual-tree method on the device, FP64: fortran/octree_default.f90
// :1095-1712 (methods 20/21/22; Dehnen 2000, with the octupole torque term of
// :1530-1557 for multipole 8).
//
// The tree is the compact octree of the build.  Entities are its nodes
// [0, M) and the bodies n + p (sorted position p); a body is a leaf with no
// extent (rmax 0), a node's children are its child nodes and lone bodies, or,
// for a node of identical keys, its bodies.
//
//  1. rmax (evaluate_rmax :1095-1131), level by level from the deepest: the
//     largest distance from a node's centre of mass to any child's centre of
//     mass plus that child's rmax (massless children skipped).
//  2. Dual traversal (mutual_interaction_walk_* :1133-1402) as a sequence of
//     generations of node pairs, starting from (root, root) of every system:
//     a pair with a massless member is dropped; (a, a) becomes the pairs of
//     a's children (i <= j; a body with itself is dropped); a pair with
//     (rmax_a + rmax_b)^2 <= theta^2 |z_a - z_b|^2 is a mutual interaction;
//     otherwise the member with the larger rmax (a on ties) is replaced by its
//     children.  Each generation is one launch over the previous one's pairs;
//     the lists live in preallocated buffers whose fill the host reads once at
//     the end, growing them and repeating when one overflowed.
//  3. Each mutual pair (a, b) becomes the two one-sided terms (a <- b) and
//     (b <- a) of :1200-1221, keyed (target, source) and radix-sorted, so every
//     target sums its terms in one fixed order (results do not depend on the
//     schedule nor on the other systems of a batch).  Term (t <- s), with
//     R = z_t - z_s (evaluate_mutual_interaction_* :1425-1558):
//       field  += M_s (D1 + Q_s : D3 / (2 M_s))      D1 = -G R r^-3
//       hess   += M_s D2,  third += M_s D3           (r^2 = R^2 + eps^2)
//       field  += (octupole) 0.5 (3 G r^-5 c - 15 G r^-7 C:RR) / M_t,
//                 C_jkl = M_s O_t,jkl - M_t O_s,jkl, c_j = C_jkk
//     which is the reference's update of both nodes written once per side.
//     Terms between coincident points without softening (r = 0) are skipped.
//  4. Downward pass (dehnen_forces :1560-1673), level by level from the root:
//     child field += parent field + H d + d.T.d / 2, child hessian += H + T d,
//     child third += T, d = child centre of mass - parent's.  A body's force is
//     m times its field.
#include "bh_internal.cuh"

namespace bh {

namespace {

constexpr int kGenerations = 2 * (kMaxDepth + 2) + 4;  // each generation deepens a pair

struct Ent {
  const int4 *meta;
  const int32_t *child;
  const double4 *com;
  const double4 *spos;
  const double *quad;
  const double *oct;
  const double *rmax;
  int64_t n;  // bodies: entity n + p is body p
};

__device__ __forceinline__ double4 ent_com(const Ent &e, int64_t i) {
  return i < e.n ? e.com[i] : e.spos[i - e.n];
}
__device__ __forceinline__ double ent_rmax(const Ent &e, int64_t i) {
  return i < e.n ? e.rmax[i] : 0.0;
}
__device__ __forceinline__ int node_nchild(int4 mt) { return mt.w > 0 ? mt.w : mt.y; }
__device__ __forceinline__ int64_t node_child(const Ent &e, int64_t j, int4 mt, int k) {
  if (mt.w > 0) {
    const int32_t c = e.child[8 * j + k];
    return c >= 0 ? (int64_t)c : e.n + (int64_t)(~c);
  }
  return e.n + mt.x + k;
}

__global__ void __launch_bounds__(128)
rmax_level_kernel(int level, const int32_t *__restrict__ level_begin, Ent e, double *rmax) {
  const int lb = level_begin[level], le = level_begin[level + 1];
  for (int j = lb + blockIdx.x * blockDim.x + threadIdx.x; j < le; j += gridDim.x * blockDim.x) {
    const int4 mt = e.meta[j];
    const double4 c = e.com[j];
    double r = 0.0;
    const int k = node_nchild(mt);
    for (int q = 0; q < k; ++q) {
      const int64_t ch = node_child(e, j, mt, q);
      const double4 cc = ent_com(e, ch);
      if (cc.w == 0.0) continue;
      const double dx = cc.x - c.x, dy = cc.y - c.y, dz = cc.z - c.z;
      const double v = sqrt(dx * dx + dy * dy + dz * dz) + ent_rmax(e, ch);
      if (v > r) r = v;
    }
    rmax[j] = r;
  }
}

__global__ void roots_frontier_kernel(const SysScalars *__restrict__ ss, int nsys, int2 *fout,
                                      unsigned long long *nout) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsys || ss[s].root < 0) return;
  const unsigned long long slot = atomicAdd(nout, 1ull);
  fout[slot] = make_int2(ss[s].root, ss[s].root);
}

__device__ __forceinline__ int64_t warp_incl_scan64(int64_t v, int lane) {
#pragma unroll
  for (int o = 1; o < kWarp; o <<= 1) {
    const int64_t t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  return v;
}

// Reserves `cnt` slots for this lane in a list shared by the grid: one atomic
// per warp on the list's counter.  Returns the lane's first slot, or -1 when
// the warp's slots would pass `cap` (the list overflowed).
__device__ __forceinline__ int64_t warp_reserve(unsigned long long *counter, int64_t cnt,
                                                int64_t cap, int lane, unsigned long long *flags,
                                                unsigned long long flag) {
  const int64_t incl = warp_incl_scan64(cnt, lane);
  const int64_t total = __shfl_sync(0xffffffffu, incl, kWarp - 1);
  int64_t base = 0;
  if (lane == kWarp - 1 && total > 0) base = (int64_t)atomicAdd(counter, (unsigned long long)total);
  base = __shfl_sync(0xffffffffu, base, kWarp - 1);
  if (total == 0) return 0;
  if (base + total > cap) {
    if (lane == kWarp - 1) atomicOr(flags, flag);
    return -1;
  }
  return base + incl - cnt;
}

// One generation of the dual traversal.  Warps go through the input pairs 32
// at a time; every lane classifies its pair, then the warp reserves the
// output slots of all its lanes at once.
__global__ void __launch_bounds__(256)
dual_step_kernel(Ent e, const int2 *__restrict__ fin, const unsigned long long *__restrict__ nin,
                 int64_t cap_in, int2 *__restrict__ fout, unsigned long long *nout, int64_t cap_out,
                 int2 *__restrict__ mut, unsigned long long *nmut, int64_t cap_mut, double theta2,
                 unsigned long long *flags) {
  // after an overflow the count exceeds what was written: read only the buffer
  const int64_t n_in = (int64_t)*nin < cap_in ? (int64_t)*nin : cap_in;
  const int lane = threadIdx.x & (kWarp - 1);
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i0 = (int64_t)blockIdx.x * blockDim.x + (threadIdx.x - lane); i0 < n_in;
       i0 += stride) {
    const int64_t i = i0 + lane;
    // kind: 0 nothing, 1 children pairs of a self pair, 2 mutual, 3 open `o`
    int kind = 0, k = 0;
    int64_t a = 0, b = 0, o = 0, other = 0;
    bool open_a = false;
    int4 mt = make_int4(0, 0, 0, 0);
    if (i < n_in) {
      a = fin[i].x; b = fin[i].y;
      const double4 ca = ent_com(e, a), cb = ent_com(e, b);
      if (ca.w != 0.0 && cb.w != 0.0) {
        if (a == b) {
          if (a < e.n) {  // a body with itself is dropped
            mt = e.meta[a];
            k = node_nchild(mt);
            kind = 1;
          }
        } else {
          const double dx = ca.x - cb.x, dy = ca.y - cb.y, dz = ca.z - cb.z;
          const double dist2 = dx * dx + dy * dy + dz * dz;
          const double ra = ent_rmax(e, a), rb = ent_rmax(e, b);
          const double rs = ra + rb;
          if (rs * rs <= theta2 * dist2) {
            kind = 2;
          } else {
            open_a = ra >= rb;
            o = open_a ? a : b;
            other = open_a ? b : a;
            if (o >= e.n) {
              atomicOr(flags, 4ull);  // cannot happen: bodies have rmax 0
            } else {
              mt = e.meta[o];
              k = node_nchild(mt);
              kind = 3;
            }
          }
        }
      }
    }
    const int64_t n_out = kind == 1 ? (int64_t)k * (k + 1) / 2 : (kind == 3 ? k : 0);
    const int64_t fo = warp_reserve(nout, n_out, cap_out, lane, flags, 1ull);
    const int64_t mo = warp_reserve(nmut, kind == 2 ? 1 : 0, cap_mut, lane, flags, 2ull);
    if (kind == 2 && mo >= 0) mut[mo] = make_int2((int)a, (int)b);
    if (kind == 1 && fo >= 0) {
      int64_t w = fo;
      for (int p = 0; p < k; ++p) {
        const int64_t cp = node_child(e, a, mt, p);
        for (int q = p; q < k; ++q) fout[w++] = make_int2((int)cp, (int)node_child(e, a, mt, q));
      }
    }
    if (kind == 3 && fo >= 0) {
      for (int q = 0; q < k; ++q) {
        const int64_t c = node_child(e, o, mt, q);
        fout[fo + q] = open_a ? make_int2((int)c, (int)other) : make_int2((int)other, (int)c);
      }
    }
  }
}

// Both one-sided terms of every mutual pair, keyed (target << eb) | source.
__global__ void __launch_bounds__(256)
expand_kernel(const int2 *__restrict__ mut, int64_t np, int eb, uint64_t *__restrict__ keys,
              int32_t *__restrict__ vals, int32_t *cnt) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < np;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t a = (uint32_t)mut[i].x, b = (uint32_t)mut[i].y;
    keys[2 * (int64_t)i] = (a << eb) | b;
    keys[2 * (int64_t)i + 1] = (b << eb) | a;
    vals[2 * (int64_t)i] = 0;
    vals[2 * (int64_t)i + 1] = 0;
    atomicAdd(&cnt[a], 1);
    atomicAdd(&cnt[b], 1);
  }
}

// One one-sided term (t <- s) added to f (3), h (6), tt (10).
template <int ORDER>
__device__ __forceinline__ void add_term(const Ent &e, int64_t t, const double4 &ct, bool tnode,
                                         int64_t s, double G, double eps2, double *f, double *h,
                                         double *tt) {
  const double4 cs = ent_com(e, s);
  const double Ms = cs.w, Mt = ct.w;
  const double dx = ct.x - cs.x, dy = ct.y - cs.y, dz = ct.z - cs.z;
  const double r2 = dx * dx + dy * dy + dz * dz + eps2;
  if (r2 == 0.0) return;
  const double rinv = 1.0 / sqrt(r2);
  const double rinv2 = rinv * rinv;
  const double rinv3 = rinv * rinv2;
  const double D1x = -G * dx * rinv3, D1y = -G * dy * rinv3, D1z = -G * dz * rinv3;
  if (ORDER < 4) {
    f[0] = f[0] + Ms * D1x; f[1] = f[1] + Ms * D1y; f[2] = f[2] + Ms * D1z;
    return;
  }
  const double rinv5 = rinv3 * rinv2, rinv7 = rinv5 * rinv2;
  double D2[6], D3[10];
  D2[0] = G * (3.0 * dx * dx * rinv5 - rinv3);
  D2[1] = G * (3.0 * dy * dy * rinv5 - rinv3);
  D2[2] = G * (3.0 * dz * dz * rinv5 - rinv3);
  D2[3] = G * 3.0 * dx * dy * rinv5;
  D2[4] = G * 3.0 * dx * dz * rinv5;
  D2[5] = G * 3.0 * dy * dz * rinv5;
  D3[0] = G * (-15.0 * dx * dx * dx * rinv7 + 9.0 * dx * rinv5);
  D3[1] = G * (-15.0 * dx * dx * dy * rinv7 + 3.0 * dy * rinv5);
  D3[2] = G * (-15.0 * dx * dx * dz * rinv7 + 3.0 * dz * rinv5);
  D3[3] = G * (-15.0 * dx * dy * dy * rinv7 + 3.0 * dx * rinv5);
  D3[4] = G * (-15.0 * dx * dy * dz * rinv7);
  D3[5] = G * (-15.0 * dx * dz * dz * rinv7 + 3.0 * dx * rinv5);
  D3[6] = G * (-15.0 * dy * dy * dy * rinv7 + 9.0 * dy * rinv5);
  D3[7] = G * (-15.0 * dy * dy * dz * rinv7 + 3.0 * dz * rinv5);
  D3[8] = G * (-15.0 * dy * dz * dz * rinv7 + 3.0 * dy * rinv5);
  D3[9] = G * (-15.0 * dz * dz * dz * rinv7 + 9.0 * dz * rinv5);
  double cq[3] = {0.0, 0.0, 0.0};
  if (s < e.n) {  // a node's specific quadrupole; a body has none
    const double *q = e.quad + 6 * s;
    const double Q0 = q[0] / Ms, Q1 = q[1] / Ms, Q2 = q[2] / Ms, Q3 = q[3] / Ms, Q4 = q[4] / Ms,
                 Q5 = q[5] / Ms;
    cq[0] = Q0 * D3[0] + 2.0 * Q3 * D3[1] + 2.0 * Q4 * D3[2] + Q1 * D3[3] + 2.0 * Q5 * D3[4] +
            Q2 * D3[5];
    cq[1] = Q0 * D3[1] + 2.0 * Q3 * D3[3] + 2.0 * Q4 * D3[4] + Q1 * D3[6] + 2.0 * Q5 * D3[7] +
            Q2 * D3[8];
    cq[2] = Q0 * D3[2] + 2.0 * Q3 * D3[4] + 2.0 * Q4 * D3[5] + Q1 * D3[7] + 2.0 * Q5 * D3[8] +
            Q2 * D3[9];
  }
  f[0] = f[0] + Ms * (D1x + 0.5 * cq[0]);
  f[1] = f[1] + Ms * (D1y + 0.5 * cq[1]);
  f[2] = f[2] + Ms * (D1z + 0.5 * cq[2]);
#pragma unroll
  for (int q = 0; q < 6; ++q) h[q] = h[q] + Ms * D2[q];
#pragma unroll
  for (int q = 0; q < 10; ++q) tt[q] = tt[q] + Ms * D3[q];
  if (ORDER >= 8 && (tnode || s < e.n)) {
    // octupole torque term (:1530-1557); a body's octupole is zero.
    // C_jkl = Ms O_t - Mt O_s, components 0 xxx 1 xyy 2 xzz 3 yxx 4 yyy 5 yzz
    // 6 zxx 7 zyy 8 zzz 9 xyz (the index map of :233-241)
    const double *ot = tnode ? e.oct + 14 * t : nullptr;
    const double *os = s < e.n ? e.oct + 14 * s : nullptr;
    double C[10];
#pragma unroll
    for (int q = 0; q < 10; ++q) C[q] = (ot ? Ms * ot[q] : 0.0) - (os ? Mt * os[q] : 0.0);
    const double cx = C[0] + C[1] + C[2], cy = C[3] + C[4] + C[5], cz = C[6] + C[7] + C[8];
    const double crx = C[0] * dx * dx + C[1] * dy * dy + C[2] * dz * dz +
                       2.0 * (C[3] * dx * dy + C[6] * dx * dz + C[9] * dy * dz);
    const double cry = C[3] * dx * dx + C[4] * dy * dy + C[5] * dz * dz +
                       2.0 * (C[1] * dx * dy + C[9] * dx * dz + C[7] * dy * dz);
    const double crz = C[6] * dx * dx + C[7] * dy * dy + C[8] * dz * dz +
                       2.0 * (C[9] * dx * dy + C[2] * dx * dz + C[5] * dy * dz);
    const double a3 = 3.0 * G * rinv5, a15 = 15.0 * G * rinv7;
    f[0] = f[0] + 0.5 * (a3 * cx - a15 * crx) / Mt;
    f[1] = f[1] + 0.5 * (a3 * cy - a15 * cry) / Mt;
    f[2] = f[2] + 0.5 * (a3 * cz - a15 * crz) / Mt;
  }
}

// Sum of the one-sided terms of every target, one warp per target: lane l
// adds terms l, l + 32, ... of the target's source-ordered list, then the
// lanes' sums are combined by a fixed butterfly, so the result depends only on
// the target's own list.
template <int ORDER>
__global__ void __launch_bounds__(128)
eval_kernel(Ent e, int64_t ne, const int32_t *__restrict__ beg, const uint64_t *__restrict__ keys,
            int eb, double G, double eps2, double *__restrict__ F, double *__restrict__ H,
            double *__restrict__ T) {
  constexpr int NV = ORDER >= 4 ? 19 : 3;
  const uint64_t mask = (1ull << eb) - 1;
  const int lane = threadIdx.x & (kWarp - 1);
  const int64_t wstride = ((int64_t)gridDim.x * blockDim.x) / kWarp;
  for (int64_t t = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / kWarp; t < ne; t += wstride) {
    double v[19];
#pragma unroll
    for (int q = 0; q < 19; ++q) v[q] = 0.0;
    const int kb = beg[t], ke = beg[t + 1];
    if (kb < ke) {
      const double4 ct = ent_com(e, t);
      const bool tnode = t < e.n;
      for (int k = kb + lane; k < ke; k += kWarp)
        add_term<ORDER>(e, t, ct, tnode, (int64_t)(keys[k] & mask), G, eps2, v, v + 3, v + 9);
#pragma unroll
      for (int q = 0; q < NV; ++q) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[q] = v[q] + __shfl_xor_sync(0xffffffffu, v[q], o);
      }
    }
    if (lane == 0) {
#pragma unroll
      for (int q = 0; q < 3; ++q) F[3 * t + q] = v[q];
      if (ORDER >= 4) {
#pragma unroll
        for (int q = 0; q < 6; ++q) H[6 * t + q] = v[3 + q];
#pragma unroll
        for (int q = 0; q < 10; ++q) T[10 * t + q] = v[9 + q];
      }
    }
  }
}

// One level of the downward pass: every node of the level pushes its field,
// hessian and third derivatives to its children.
template <int ORDER>
__global__ void __launch_bounds__(128)
down_level_kernel(int level, const int32_t *__restrict__ level_begin, Ent e, double *F, double *H,
                  double *T) {
  const int lb = level_begin[level], le = level_begin[level + 1];
  for (int j = lb + blockIdx.x * blockDim.x + threadIdx.x; j < le; j += gridDim.x * blockDim.x) {
    const int4 mt = e.meta[j];
    const double4 cj = e.com[j];
    const double Fx = F[3 * j], Fy = F[3 * j + 1], Fz = F[3 * j + 2];
    double h[6], t[10];
    if (ORDER >= 4) {
#pragma unroll
      for (int q = 0; q < 6; ++q) h[q] = H[6 * (int64_t)j + q];
#pragma unroll
      for (int q = 0; q < 10; ++q) t[q] = T[10 * (int64_t)j + q];
    }
    const int k = node_nchild(mt);
    for (int q = 0; q < k; ++q) {
      const int64_t c = node_child(e, j, mt, q);
      const double4 cc = ent_com(e, c);
      if (cc.w == 0.0) continue;
      double fx = F[3 * c] + Fx, fy = F[3 * c + 1] + Fy, fz = F[3 * c + 2] + Fz;
      if (ORDER >= 4) {
        const double dx = cc.x - cj.x, dy = cc.y - cj.y, dz = cc.z - cj.z;
        const double hxx = h[0], hyy = h[1], hzz = h[2], hxy = h[3], hxz = h[4], hyz = h[5];
        const double txxx = t[0], txxy = t[1], txxz = t[2], txyy = t[3], txyz = t[4], txzz = t[5],
                     tyyy = t[6], tyyz = t[7], tyzz = t[8], tzzz = t[9];
        fx = fx + hxx * dx + hxy * dy + hxz * dz + txxy * dx * dy + txxz * dx * dz + txyz * dy * dz +
             0.5 * (txxx * dx * dx + txyy * dy * dy + txzz * dz * dz);
        fy = fy + hxy * dx + hyy * dy + hyz * dz + txyy * dx * dy + txyz * dx * dz + tyyz * dy * dz +
             0.5 * (txxy * dx * dx + tyyy * dy * dy + tyzz * dz * dz);
        fz = fz + hxz * dx + hyz * dy + hzz * dz + txyz * dx * dy + txzz * dx * dz + tyzz * dy * dz +
             0.5 * (txxz * dx * dx + tyyz * dy * dy + tzzz * dz * dz);
        if (c < e.n) {
          double *hc = H + 6 * c;
          hc[0] = hc[0] + hxx + txxx * dx + txxy * dy + txxz * dz;
          hc[1] = hc[1] + hyy + txyy * dx + tyyy * dy + tyyz * dz;
          hc[2] = hc[2] + hzz + txzz * dx + tyzz * dy + tzzz * dz;
          hc[3] = hc[3] + hxy + txxy * dx + txyy * dy + txyz * dz;
          hc[4] = hc[4] + hxz + txxz * dx + txyz * dy + txzz * dz;
          hc[5] = hc[5] + hyz + txyz * dx + tyyz * dy + tyzz * dz;
          double *tc = T + 10 * c;
#pragma unroll
          for (int r = 0; r < 10; ++r) tc[r] = tc[r] + t[r];
        }
      }
      F[3 * c] = fx; F[3 * c + 1] = fy; F[3 * c + 2] = fz;
    }
  }
}

// Forces in the original order, one (n_s, 3) Fortran block per system.
__global__ void __launch_bounds__(256)
dehnen_out_kernel(int64_t n, const double *__restrict__ F, const double4 *__restrict__ spos,
                  const int32_t *__restrict__ perm, const int32_t *__restrict__ sys_of,
                  const SysScalars *__restrict__ ss, int out_kind, double *__restrict__ out) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x) {
    const SysScalars &s = ss[sys_of[p]];
    const double sc = out_kind == 0 ? spos[p].w : 1.0;
    const int64_t o = perm[p] - s.off;
    double *base = out + 3 * s.off;
    const double *f = F + 3 * (n + p);
    base[o] = sc * f[0];
    base[s.n + o] = sc * f[1];
    base[2 * s.n + o] = sc * f[2];
  }
}

template <typename T>
cudaError_t grow(T *&p, int64_t &cap, int64_t need) {
  if (p && cap >= need) return cudaSuccess;
  if (p) cudaFree(p);
  p = nullptr;
  cap = 0;
  const cudaError_t e = cudaMalloc((void **)&p, (size_t)need * sizeof(T));
  if (e == cudaSuccess) cap = need;
  return e;
}

int bits_for64(int64_t v) {
  int b = 1;
  while (((int64_t)1 << b) <= v) ++b;
  return b;
}

}  // namespace

void free_dehnen(DehnenBuffers &d) {
  void *ptrs[] = {d.rmax, d.F, d.H, d.T, d.front, d.mut, d.keys, d.vals, d.cnt, d.beg, d.hist,
                  d.scan_tmp, d.counters};
  for (void *q : ptrs)
    if (q) cudaFree(q);
  d = DehnenBuffers();
}

int run_dehnen(int64_t n, const WalkParams &p, Buffers &b, DehnenBuffers &d, double *out,
               cudaStream_t s) {
  const int64_t ne = 2 * n;
  if (grow(d.rmax, d.rmax_cap, n) != cudaSuccess) return 1;
  if (grow(d.F, d.F_cap, 3 * ne) != cudaSuccess) return 1;
  if (p.order >= 4 && grow(d.H, d.H_cap, 6 * ne) != cudaSuccess) return 1;
  if (p.order >= 4 && grow(d.T, d.T_cap, 10 * ne) != cudaSuccess) return 1;
  if (grow(d.cnt, d.cnt_cap, ne + 1) != cudaSuccess) return 1;
  if (grow(d.beg, d.beg_cap, ne + 1) != cudaSuccess) return 1;
  if (grow(d.scan_tmp, d.scan_tmp_cap, scan_tmp_entries(ne + 1)) != cudaSuccess) return 1;
  if (grow(d.counters, d.counters_cap, 8) != cudaSuccess) return 1;
  if (d.front_cap < 2 * 16 * n) d.want_front = 16 * n;  // per generation, either buffer
  if (d.mut_cap < 32 * n) d.want_mut = 32 * n;

  Ent e;
  e.meta = b.cn_meta; e.child = b.cn_child; e.com = b.cn_com; e.spos = b.spos;
  e.quad = b.cn_quad; e.oct = b.cn_oct; e.rmax = d.rmax; e.n = n;
  const int lgrid = grid_for(n / 2 + 1, 128, 148 * 8);
  for (int level = kMaxDepth; level >= 0; --level)
    rmax_level_kernel<<<lgrid, 128, 0, s>>>(level, b.level_begin, e, d.rmax);

  const int eb = bits_for64(ne);
  // counters: [0], [1] frontier sizes, [2] mutual pairs, [3] overflow flags
  unsigned long long *cnt_front = d.counters;
  unsigned long long h[4] = {0, 0, 0, 0};
  for (int attempt = 0; attempt < 8; ++attempt) {
    if (grow(d.front, d.front_cap, 2 * d.want_front) != cudaSuccess) return 1;
    if (grow(d.mut, d.mut_cap, d.want_mut) != cudaSuccess) return 1;
    int2 *f0 = d.front, *f1 = d.front + d.front_cap / 2;
    const int64_t fcap = d.front_cap / 2;
    cudaMemsetAsync(d.counters, 0, 8 * sizeof(unsigned long long), s);
    roots_frontier_kernel<<<(b.nsys + 127) / 128, 128, 0, s>>>(b.ss, b.nsys, f0, cnt_front);
    for (int g = 0; g < kGenerations; ++g) {
      int2 *fi = (g & 1) ? f1 : f0, *fo = (g & 1) ? f0 : f1;
      unsigned long long *ni = cnt_front + (g & 1), *no = cnt_front + ((g + 1) & 1);
      cudaMemsetAsync(no, 0, sizeof(unsigned long long), s);
      dual_step_kernel<<<148 * 8, 256, 0, s>>>(e, fi, ni, fcap, fo, no, fcap, d.mut, cnt_front + 2,
                                               d.mut_cap, p.theta2, cnt_front + 3);
    }
    if (cudaMemcpyAsync(h, d.counters, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                        s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
      return 2;
    if (h[3] & 4) return 3;
    const bool more_front = (h[3] & 1) != 0, more_mut = (h[3] & 2) != 0;
    if (!more_front && !more_mut) {
      if (h[kGenerations & 1] != 0) return 3;  // the traversal did not close
      break;
    }
    if (attempt == 7) return 4;
    if (more_front) d.want_front *= 2;
    if (more_mut) d.want_mut *= 2;
    if (d.want_mut > ((int64_t)1 << 30) || d.want_front > ((int64_t)1 << 30)) return 4;
  }
  const int64_t np = (int64_t)h[2];
  const int64_t nh = 2 * np;
  if (grow(d.keys, d.keys_cap, 2 * (nh > 0 ? nh : 1)) != cudaSuccess) return 1;
  if (grow(d.vals, d.vals_cap, 2 * (nh > 0 ? nh : 1)) != cudaSuccess) return 1;
  if (grow(d.hist, d.hist_cap, radix_hist_entries(nh > 0 ? nh : 1)) != cudaSuccess) return 1;
  cudaMemsetAsync(d.cnt, 0, (ne + 1) * sizeof(int32_t), s);
  if (np > 0) {
    const int g = grid_for(np, 256, 148 * 16);
    expand_kernel<<<g, 256, 0, s>>>(d.mut, np, eb, d.keys, d.vals, d.cnt);
    radix_sort_pairs(d.keys, d.vals, d.keys + nh, d.vals + nh, nh, nullptr, 2 * eb, d.hist,
                     &b.sc->err, s);
  }
  exclusive_scan(d.cnt, d.beg, ne + 1, nullptr, nullptr, d.scan_tmp, s);
  const int egrid = grid_for(ne * kWarp, 128, 148 * 32);
  const double G = p.G, eps2 = p.eps2;
  if (p.order >= 8)
    eval_kernel<8><<<egrid, 128, 0, s>>>(e, ne, d.beg, d.keys, eb, G, eps2, d.F, d.H, d.T);
  else if (p.order >= 4)
    eval_kernel<4><<<egrid, 128, 0, s>>>(e, ne, d.beg, d.keys, eb, G, eps2, d.F, d.H, d.T);
  else
    eval_kernel<1><<<egrid, 128, 0, s>>>(e, ne, d.beg, d.keys, eb, G, eps2, d.F, d.H, d.T);
  for (int level = 0; level <= kMaxDepth; ++level) {
    if (p.order >= 4)
      down_level_kernel<4><<<lgrid, 128, 0, s>>>(level, b.level_begin, e, d.F, d.H, d.T);
    else
      down_level_kernel<1><<<lgrid, 128, 0, s>>>(level, b.level_begin, e, d.F, d.H, d.T);
  }
  dehnen_out_kernel<<<grid_for(n, 256, 148 * 16), 256, 0, s>>>(n, d.F, b.spos, b.v0, b.sys_of,
                                                                 b.ss, p.out_kind, out);
  d.pairs = np;
  return 0;
}

}  // namespace bh
