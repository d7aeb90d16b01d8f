// Upward pass: mass, centre of mass, quadrupole and octupole of every octree
// node, level by level from the deepest level to the root, in FP64.
//
// Follows the translation method of fortran/octree_default.f90:744-882
// (evaluate_multipole): the node's mass and centre of mass from its children
// (:782-799); for every child, first its own moments (:815-821), then the
// parallel-axis terms m d d (:823-828) and m d d d (:830-844), then the
// octupole cross terms 3 d Q of a child node (:846-872); finally the summary
// sums oct(11) = sum 1..10, oct(12..14) = row sums (:875-880).  Moments are raw
// (not trace-free) moments about the node's centre of mass: quad = xx yy zz xy
// xz yz; oct = xxx xyy xzz yxx yyy yzz zxx zyy zzz xyz (the reference's order).
// Lone particles are point children (mass, position, no moments), so a node's
// children are processed exactly like the reference's twig/leaf children.
//
// The same pass writes the normalised FP32 copies used by the FP32 walk:
// quadrupole / (M ssa^2) with its trace, octupole / (M ssa^3), where M is the
// total mass and ssa the root cube side, so the walk's values are O(1)
// whatever the physical units.
#include "bh_internal.cuh"

namespace bh {

namespace {

template <int ORDER>
__global__ void __launch_bounds__(128)
upward_level_kernel(int level, const int32_t *__restrict__ level_begin,
                    const int4 *__restrict__ meta, const int32_t *__restrict__ child,
                    const double4 *__restrict__ spos, const int32_t *__restrict__ sys_of,
                    const SysScalars *__restrict__ sys,
                    double4 *__restrict__ com, double *__restrict__ quad,
                    double *__restrict__ oct, float4 *__restrict__ fq, float4 *__restrict__ fo) {
  const int lb = level_begin[level], le = level_begin[level + 1];
  for (int j = lb + blockIdx.x * blockDim.x + threadIdx.x; j < le; j += gridDim.x * blockDim.x) {
    const int4 mt = meta[j];  // first, count, level, nchild
    const SysScalars &ss = sys[sys_of[mt.x]];
    const double inv_m = 1.0 / ss.mass;
    const double inv_s = 1.0 / ss.ssa;
    const double nq = inv_m * inv_s * inv_s, no = nq * inv_s;
    const bool bucket = (mt.w == 0);
    const int nch = bucket ? mt.y : mt.w;
    // pass 1: mass and centre of mass
    double M = 0.0, cx = 0.0, cy = 0.0, cz = 0.0;
    for (int c = 0; c < nch; ++c) {
      double cm, px, py, pz;
      if (bucket) {
        double4 p = spos[mt.x + c];
        cm = p.w; px = p.x; py = p.y; pz = p.z;
      } else {
        int32_t ch = child[8 * j + c];
        if (ch < 0) {
          double4 p = spos[~ch];
          cm = p.w; px = p.x; py = p.y; pz = p.z;
        } else {
          double4 q = com[ch];
          cm = q.w; px = q.x; py = q.y; pz = q.z;
        }
      }
      M = M + cm;
      cx = cx + cm * px;
      cy = cy + cm * py;
      cz = cz + cm * pz;
    }
    cx = cx / M; cy = cy / M; cz = cz / M;
    com[j] = make_double4(cx, cy, cz, M);
    if (ORDER < 4) continue;
    // pass 2: moments about (cx, cy, cz)
    double Q[6] = {0, 0, 0, 0, 0, 0};
    double O[14] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int c = 0; c < nch; ++c) {
      double pm, px, py, pz;
      int32_t node = -1;
      if (bucket) {
        double4 p = spos[mt.x + c];
        pm = p.w; px = p.x; py = p.y; pz = p.z;
      } else {
        int32_t ch = child[8 * j + c];
        if (ch < 0) {
          double4 p = spos[~ch];
          pm = p.w; px = p.x; py = p.y; pz = p.z;
        } else {
          double4 q = com[ch];
          pm = q.w; px = q.x; py = q.y; pz = q.z;
          node = ch;
        }
      }
      const double dx = px - cx, dy = py - cy, dz = pz - cz;
      double Qd[6];
      if (node >= 0) {
#pragma unroll
        for (int k = 0; k < 6; ++k) { Qd[k] = quad[6 * (int64_t)node + k]; Q[k] = Q[k] + Qd[k]; }
        if (ORDER >= 8) {
#pragma unroll
          for (int k = 0; k < 14; ++k) O[k] = O[k] + oct[14 * (int64_t)node + k];
        }
      }
      Q[0] = Q[0] + pm * (dx * dx);
      Q[1] = Q[1] + pm * (dy * dy);
      Q[2] = Q[2] + pm * (dz * dz);
      Q[3] = Q[3] + pm * dx * dy;
      Q[4] = Q[4] + pm * dx * dz;
      Q[5] = Q[5] + pm * dy * dz;
      if (ORDER >= 8) {
        O[0] = O[0] + pm * dx * (dx * dx);
        O[1] = O[1] + pm * dx * (dy * dy);
        O[2] = O[2] + pm * dx * (dz * dz);
        O[3] = O[3] + pm * dy * (dx * dx);
        O[4] = O[4] + pm * dy * (dy * dy);
        O[5] = O[5] + pm * dy * (dz * dz);
        O[6] = O[6] + pm * dz * (dx * dx);
        O[7] = O[7] + pm * dz * (dy * dy);
        O[8] = O[8] + pm * dz * (dz * dz);
        O[9] = O[9] + pm * dx * dy * dz;
        if (node >= 0) {
          O[0] = O[0] + 3.0 * dx * Qd[0];
          O[1] = O[1] + 2.0 * dy * Qd[3] + dx * Qd[1];
          O[2] = O[2] + 2.0 * dz * Qd[4] + dx * Qd[2];
          O[3] = O[3] + 2.0 * dx * Qd[3] + dy * Qd[0];
          O[4] = O[4] + 3.0 * dy * Qd[1];
          O[5] = O[5] + 2.0 * dz * Qd[5] + dy * Qd[2];
          O[6] = O[6] + 2.0 * dx * Qd[4] + dz * Qd[0];
          O[7] = O[7] + 2.0 * dy * Qd[5] + dz * Qd[1];
          O[8] = O[8] + 3.0 * dz * Qd[2];
          O[9] = O[9] + dx * Qd[5] + dy * Qd[4] + dz * Qd[3];
        }
      }
    }
#pragma unroll
    for (int k = 0; k < 6; ++k) quad[6 * (int64_t)j + k] = Q[k];
    const double trq = Q[0] + Q[1] + Q[2];
    fq[2 * (int64_t)j] = make_float4((float)(Q[0] * nq), (float)(Q[1] * nq), (float)(Q[2] * nq),
                                     (float)(Q[3] * nq));
    fq[2 * (int64_t)j + 1] =
        make_float4((float)(Q[4] * nq), (float)(Q[5] * nq), (float)(trq * nq), 0.0f);
    if (ORDER >= 8) {
      double s = 0.0;
#pragma unroll
      for (int k = 0; k < 10; ++k) s = s + O[k];
      O[10] = s;
      O[11] = O[0] + O[1] + O[2];
      O[12] = O[3] + O[4] + O[5];
      O[13] = O[6] + O[7] + O[8];
#pragma unroll
      for (int k = 0; k < 14; ++k) oct[14 * (int64_t)j + k] = O[k];
      float4 *f = fo + 4 * (int64_t)j;
      f[0] = make_float4((float)(O[0] * no), (float)(O[1] * no), (float)(O[2] * no), (float)(O[3] * no));
      f[1] = make_float4((float)(O[4] * no), (float)(O[5] * no), (float)(O[6] * no), (float)(O[7] * no));
      f[2] = make_float4((float)(O[8] * no), (float)(O[9] * no), (float)(O[11] * no), (float)(O[12] * no));
      f[3] = make_float4((float)(O[13] * no), 0.0f, 0.0f, 0.0f);
    }
  }
}

}  // namespace

void launch_upward(int64_t n, int L, int order, Buffers &b, cudaStream_t s) {
  (void)L;
  const int grid = grid_for(n / 2 + 1, 128, 148 * 8);
  for (int level = kMaxDepth; level >= 0; --level) {
    if (order >= 8)
      upward_level_kernel<8><<<grid, 128, 0, s>>>(level, b.level_begin, b.cn_meta, b.cn_child,
                                                  b.spos, b.sys_of, b.ss, b.cn_com, b.cn_quad, b.cn_oct,
                                                  b.cn_fq, b.cn_fo);
    else if (order >= 4)
      upward_level_kernel<4><<<grid, 128, 0, s>>>(level, b.level_begin, b.cn_meta, b.cn_child,
                                                  b.spos, b.sys_of, b.ss, b.cn_com, b.cn_quad, b.cn_oct,
                                                  b.cn_fq, b.cn_fo);
    else
      upward_level_kernel<1><<<grid, 128, 0, s>>>(level, b.level_begin, b.cn_meta, b.cn_child,
                                                  b.spos, b.sys_of, b.ss, b.cn_com, b.cn_quad, b.cn_oct,
                                                  b.cn_fq, b.cn_fo);
  }
}

}  // namespace bh
