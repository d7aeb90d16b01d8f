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
// One launch per level, deepest first; a thread computes one node, loading
// all of its child records before using any so that the loads overlap.  A
// single bottom-up launch (a per-node arrival counter, the last child's
// thread going on with the parent) gives the same bits but measured slower:
// the whole build of a 2^20-body Hernquist system took 0.90-0.93 ms with it
// (four block shapes) against 0.85 ms with these 22 launches, because each
// thread's chain of dependent node loads up the tree serialises more than the
// level launches do.  Small builds (a cooperative grid of at most half the
// resident blocks, systems up to about 37,000 bodies) run all levels in one
// cooperative launch with a grid barrier per level instead: there the level
// launches cost more than their work.  At 2^20 the cooperative launch took
// the build from 0.817 to 0.780 ms but cost the served rate 1 % (187.7 ->
// 185.8 M forces/s): a cooperative grid waits until all of it fits, so it no
// longer slips into the SMs that another lane's walk frees at its end.
//
// The same pass writes the normalised FP32 copies used by the FP32 walk:
// quadrupole / (M ssa^2) with its trace, octupole / (M ssa^3), where M is the
// total mass and ssa the root cube side, so the walk's values are O(1)
// whatever the physical units.
#include <cooperative_groups.h>

#include "bh_internal.cuh"

namespace cg = cooperative_groups;

namespace bh {

namespace {

__device__ __forceinline__ double4 ld_com(const double4 *p) {
  const double2 a = __ldcg(reinterpret_cast<const double2 *>(p));
  const double2 b = __ldcg(reinterpret_cast<const double2 *>(p) + 1);
  return make_double4(a.x, a.y, b.x, b.y);
}

// One child's contribution to the moments about (cx, cy, cz): its own
// moments (node children), then the parallel-axis and octupole cross terms.
template <int ORDER>
__device__ __forceinline__ void add_child(double pm, double px, double py, double pz, bool node,
                                          const double *Qd, const double *Od, double cx,
                                          double cy, double cz, double *Q, double *O) {
  const double dx = px - cx, dy = py - cy, dz = pz - cz;
  if (node) {
#pragma unroll
    for (int k = 0; k < 6; ++k) Q[k] = Q[k] + Qd[k];
    if (ORDER >= 8) {
#pragma unroll
      for (int k = 0; k < 14; ++k) O[k] = O[k] + Od[k];
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
    if (node) {
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

// Mass, centre of mass and moments of node j from its children.  For a node
// with child entries, all child records are loaded before any is used, so the
// loads overlap; the sums run in child order either way.
template <int ORDER>
__device__ void compute_node(int j, const int4 *__restrict__ meta, const int32_t *__restrict__ child,
                             const double4 *__restrict__ spos, const int32_t *__restrict__ sys_of,
                             const SysScalars *__restrict__ sys, double4 *com, double *quad,
                             double *oct, float4 *__restrict__ fq, float4 *__restrict__ fo) {
  const int4 mt = meta[j];  // first, count, level, nchild
  const SysScalars &ss = sys[sys_of[mt.x]];
  const double inv_m = 1.0 / ss.mass;
  const double inv_s = 1.0 / ss.ssa;
  const double nq = inv_m * inv_s * inv_s, no = nq * inv_s;
  double M = 0.0, cx = 0.0, cy = 0.0, cz = 0.0;
  double Q[6] = {0, 0, 0, 0, 0, 0};
  double O[14] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  if (mt.w == 0) {  // bucket of identical keys: its bodies are the children
    for (int c = 0; c < mt.y; ++c) {
      const double4 p = spos[mt.x + c];
      M = M + p.w;
      cx = cx + p.w * p.x;
      cy = cy + p.w * p.y;
      cz = cz + p.w * p.z;
    }
    if (M == 0.0) {  // massless node: a finite centre (it only enters sums times 0)
      const double4 p = spos[mt.x];
      cx = p.x; cy = p.y; cz = p.z;
    } else {
      cx = cx / M; cy = cy / M; cz = cz / M;
    }
    com[j] = make_double4(cx, cy, cz, M);
    if constexpr (ORDER < 4) {
      return;
    } else {
      for (int c = 0; c < mt.y; ++c) {
        const double4 p = spos[mt.x + c];
        add_child<ORDER>(p.w, p.x, p.y, p.z, false, nullptr, nullptr, cx, cy, cz, Q, O);
      }
    }
  } else {
    const int4 c0 = *reinterpret_cast<const int4 *>(child + 8 * (int64_t)j);
    const int4 c1 = *reinterpret_cast<const int4 *>(child + 8 * (int64_t)j + 4);
    const int32_t ch[8] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w};
    double4 cd[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      cd[c] = make_double4(0.0, 0.0, 0.0, 0.0);
      if (c < mt.w) cd[c] = ch[c] < 0 ? spos[~ch[c]] : ld_com(com + ch[c]);
    }
    double Qd[ORDER >= 4 ? 8 : 1][6];
    if (ORDER >= 4) {
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        if (c < mt.w && ch[c] >= 0) {
          const double2 *q2 = reinterpret_cast<const double2 *>(quad + 6 * (int64_t)ch[c]);
          const double2 a = __ldcg(q2), b = __ldcg(q2 + 1), e = __ldcg(q2 + 2);
          Qd[c][0] = a.x; Qd[c][1] = a.y; Qd[c][2] = b.x; Qd[c][3] = b.y; Qd[c][4] = e.x; Qd[c][5] = e.y;
        }
      }
    }
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      if (c < mt.w) {
        M = M + cd[c].w;
        cx = cx + cd[c].w * cd[c].x;
        cy = cy + cd[c].w * cd[c].y;
        cz = cz + cd[c].w * cd[c].z;
      }
    }
    if (M == 0.0) {  // massless node: a finite centre (it only enters sums times 0)
      cx = cd[0].x; cy = cd[0].y; cz = cd[0].z;
    } else {
      cx = cx / M; cy = cy / M; cz = cz / M;
    }
    com[j] = make_double4(cx, cy, cz, M);
    if constexpr (ORDER < 4) {
      return;
    } else {
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        if (c < mt.w) {
          double Od[14];
          if (ORDER >= 8 && ch[c] >= 0) {
#pragma unroll
            for (int k = 0; k < 14; ++k) Od[k] = __ldcg(oct + 14 * (int64_t)ch[c] + k);
          }
          add_child<ORDER>(cd[c].w, cd[c].x, cd[c].y, cd[c].z, ch[c] >= 0, Qd[c], Od, cx, cy, cz,
                           Q, O);
        }
      }
    }
  }
  if constexpr (ORDER >= 4) {
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

template <int ORDER>
__global__ void __launch_bounds__(128)
upward_level_kernel(int level, const int32_t *__restrict__ level_begin,
                    const int4 *__restrict__ meta, const int32_t *__restrict__ child,
                    const double4 *__restrict__ spos, const int32_t *__restrict__ sys_of,
                    const SysScalars *__restrict__ sys, double4 *com, double *quad, double *oct,
                    float4 *__restrict__ fq, float4 *__restrict__ fo) {
  const int lb = level_begin[level], le = level_begin[level + 1];
  for (int j = lb + blockIdx.x * blockDim.x + threadIdx.x; j < le; j += gridDim.x * blockDim.x)
    compute_node<ORDER>(j, meta, child, spos, sys_of, sys, com, quad, oct, fq, fo);
}

// All levels in one cooperative launch: the grid takes every level's nodes
// in turn, deepest first, with a grid-wide barrier after each level that has
// nodes (the barrier also makes the level's writes visible to the next one,
// which reads them through L2).  Same per-node arithmetic, so the same bits as
// the per-level launches.
template <int ORDER>
__global__ void __launch_bounds__(128)
upward_coop_kernel(const int32_t *__restrict__ level_begin, const int4 *__restrict__ meta,
                   const int32_t *__restrict__ child, const double4 *__restrict__ spos,
                   const int32_t *__restrict__ sys_of, const SysScalars *__restrict__ sys,
                   double4 *com, double *quad, double *oct, float4 *__restrict__ fq,
                   float4 *__restrict__ fo) {
  cg::grid_group grid = cg::this_grid();
  for (int level = kMaxDepth; level >= 0; --level) {
    const int lb = level_begin[level], le = level_begin[level + 1];
    if (lb >= le) continue;  // the same for every thread: no writes, no barrier
    for (int j = lb + blockIdx.x * blockDim.x + threadIdx.x; j < le; j += gridDim.x * blockDim.x)
      compute_node<ORDER>(j, meta, child, spos, sys_of, sys, com, quad, oct, fq, fo);
    if (level > 0) grid.sync();
  }
}

// Blocks of the cooperative launch that fit on the device at once (0: no
// cooperative launch here), per device and order.
template <int ORDER>
int coop_blocks() {
  static int per_dev[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 0;
  if (per_dev[dev] == 0) {
    int coop = 0, sms = 0, per_sm = 0;
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, upward_coop_kernel<ORDER>, 128, 0);
    per_dev[dev] = (coop && sms > 0 && per_sm > 0) ? per_sm * sms : -1;
  }
  return per_dev[dev] > 0 ? per_dev[dev] : 0;
}

template <int ORDER>
bool launch_upward_coop(int64_t n, Buffers &b, cudaStream_t s) {
  // inside a graph capture the level launches cost little (the graph launches
  // them back to back), and a graph holding a cooperative node is slower to
  // set up: keep the per-level form there
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone)
    return false;
  const int resident = coop_blocks<ORDER>();
  if (resident <= 0) return false;
  const int grid = grid_for(n / 2 + 1, 128, resident);
  // a cooperative grid starts only when all of it fits: keep it to small
  // builds, whose 22 level launches cost more than their work, and leave the
  // large ones (which another stream's walk shares the GPU with) per level
  if (2 * grid > resident) return false;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3(128);
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, upward_coop_kernel<ORDER>, (const int32_t *)b.level_begin,
                            (const int4 *)b.cn_meta, (const int32_t *)b.cn_child,
                            (const double4 *)b.spos, (const int32_t *)b.sys_of,
                            (const SysScalars *)b.ss, b.cn_com, b.cn_quad, b.cn_oct, b.cn_fq,
                            b.cn_fo) == cudaSuccess;
}

}  // namespace

void launch_upward(int64_t n, int L, int order, Buffers &b, cudaStream_t s) {
  (void)L;
  if (order >= 8 ? launch_upward_coop<8>(n, b, s)
                 : (order >= 4 ? launch_upward_coop<4>(n, b, s) : launch_upward_coop<1>(n, b, s)))
    return;
  cudaGetLastError();  // a refused cooperative launch: the per-level launches instead
  const int grid = grid_for(n / 2 + 1, 128, 148 * 8);
  for (int level = kMaxDepth; level >= 0; --level) {
    if (order >= 8)
      upward_level_kernel<8><<<grid, 128, 0, s>>>(level, b.level_begin, b.cn_meta, b.cn_child, b.spos,
                                                  b.sys_of, b.ss, b.cn_com, b.cn_quad, b.cn_oct,
                                                  b.cn_fq, b.cn_fo);
    else if (order >= 4)
      upward_level_kernel<4><<<grid, 128, 0, s>>>(level, b.level_begin, b.cn_meta, b.cn_child, b.spos,
                                                  b.sys_of, b.ss, b.cn_com, b.cn_quad, b.cn_oct,
                                                  b.cn_fq, b.cn_fo);
    else
      upward_level_kernel<1><<<grid, 128, 0, s>>>(level, b.level_begin, b.cn_meta, b.cn_child, b.spos,
                                                  b.sys_of, b.ss, b.cn_com, b.cn_quad, b.cn_oct,
                                                  b.cn_fq, b.cn_fo);
  }
}

}  // namespace bh
