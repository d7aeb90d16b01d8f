// Tree walks.
//
// 1. Group walk (the production path), after Barnes (1990) as restated by
//    fortran/octree_default.f90:1811-2095 (forces_groups / group_worker): one
//    warp per group of <= 64 Morton-contiguous targets.  The warp walks the
//    tree 32 nodes at a time from a per-warp stack, tests each node with the
//    box-distance MAC of :1927-1936 (size^2 <= theta^2 * dist^2 from the
//    node's centre of mass to the group's bounding box), queues accepted
//    nodes as cells and the bodies of opened leaves / lone particles as
//    bodies, and evaluates the queues in batches of 32: lane j stages entry j
//    (a coalesced load) into shared memory and every lane then sweeps the 32
//    staged entries (broadcast reads) for its own 1 or 2 targets.  Each batch
//    is summed in registers and Kahan-added (Kahan 1965) into the per-target
//    accumulator.  Positions are taken relative to the group's centre in FP64
//    and only then rounded, and everything is scaled to the root cube side and
//    total mass, so the FP32 arithmetic sees O(1) numbers.  The cell formulas
//    are the reference's (:1993-2083) with r^-3 factored out so that no
//    intermediate power of r overflows FP32.
//    Because the box distance never exceeds a member's own distance, every
//    accepted cell also passes the per-target MAC of the classic walk.
//
// 2. Reference walk: one thread per target with the semantics of
//    fortran/morton/morton_octree.f90:627-766 (barnes_hut) in FP64 over the
//    compact tree: the node containing the target is always opened, cells are
//    tested with the target-to-centre distance, lone particles are monopoles
//    at m*q/m, level-L leaves are summed particle by particle.  Used to check
//    the tree against the reference and to count the reference's interactions.
#include <math.h>

#include "bh_internal.cuh"

namespace bh {

namespace {

// The walk runs one warp per block.  The FP32 walk is compiled for 16 resident
// blocks per SM (128 registers a thread).
constexpr int kWalkBlocksPerSm = 16;
// One-warp blocks per SM the walk is compiled for, FP64 as FP32: 16 (128
// registers) against the compiler's own choice for FP64 (182 / 222 registers,
// 11 / 9 warps per SM) took the FP64 walk at 2^20 from 15.5 to 12.3 ms
// (quadrupole) and from 29.4 to 26.3 ms (octupole, despite 592 bytes of
// spills; 12 blocks: 27.1 ms), the same bits.
template <typename T, int ORDER> constexpr int walk_min_blocks() { return kWalkBlocksPerSm; }
constexpr int kCellQ = 64;
constexpr int kBodyPerLane = 16;
constexpr int kBodyQ = 32 + kWarp * kBodyPerLane;  // 544
constexpr unsigned kFull = 0xffffffffu;

template <typename T> struct Ops;
template <> struct Ops<float> {
  static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
  static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
  static __device__ __forceinline__ float rsq(float r2) { return r2 > 0.0f ? rsqrtf(r2) : 0.0f; }
};
template <> struct Ops<double> {
  static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
  static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
  static __device__ __forceinline__ double rsq(double r2) { return r2 > 0.0 ? rsqrt(r2) : 0.0; }
};

template <typename T>
__device__ __forceinline__ void kahan_add(T &s, T &c, T x) {
  T y = Ops<T>::sub(x, c);
  T t = Ops<T>::add(s, y);
  c = Ops<T>::sub(Ops<T>::sub(t, s), y);
  s = t;
}

template <int ORDER> struct StageWords { static constexpr int value = ORDER >= 8 ? 24 : (ORDER >= 4 ? 12 : 4); };

template <typename T, int ORDER>
struct __align__(16) WarpSmem {
  T stage[kWarp * StageWords<ORDER>::value];
  int cellq[kCellQ];
  int bodyq[kBodyQ];
};

struct WalkArgs {
  const int4 *meta;
  const int32_t *child;
  const double4 *com;
  const double *quad;
  const double *oct;
  const float4 *fq;
  const float4 *fo;
  const double4 *spos;
  const int32_t *perm;
  const int32_t *g_first;
  const int32_t *sys_of;
  const SysScalars *ss;
  Scalars *sc;
  int32_t *cursor;
  int32_t *stack;
  int64_t stack_cap;
  int64_t slots;
  unsigned long long *stats;
  double *out;
  int64_t n;
  double theta2, G, eps2;
  int out_kind, leaf_cap, count_stats, mac;
  int g_begin, g_end;  // groups walked: [g_begin, g_end), g_end < 0 = all
  int pipeline;        // FP32: producer/consumer warp teams
};

template <typename T>
__device__ __forceinline__ T warp_min(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(kFull, v, o));
  return v;
}
template <typename T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(kFull, v, o));
  return v;
}

__device__ __forceinline__ int warp_excl_scan(int v, int lane, int &total) {
  int x = v;
#pragma unroll
  for (int o = 1; o < kWarp; o <<= 1) {
    int t = __shfl_up_sync(kFull, x, o);
    if (lane >= o) x += t;
  }
  total = __shfl_sync(kFull, x, kWarp - 1);
  return x - v;
}

// Stage one cell (node j) as T words, all in the group's frame (positions
// relative to the group centre over the root cube side, masses over the total
// mass):
//   [0..3]   x, y, z, m
//   [4..7]   7.5 Qxx, 7.5 Qyy, 7.5 Qzz, 7.5 Qxy
//   [8..11]  7.5 Qxz, 7.5 Qyz, -1.5 trQ, O14
//   [12..23] O1..O10, O12, O13     (octupole only)
// The factors 7.5 and -1.5 of the reference's cell formula
// (octree_default.f90:2024-2027) are folded in here once per staged cell.
// Word k goes to w[k * STR]: STR = 1 for the FP64 walk, 2 for the paired FP32
// walk, whose stage holds cells 2i and 2i+1 interleaved word by word.
template <typename T, int ORDER, int STR = 1>
__device__ __forceinline__ void stage_cell(T *w, int j, const WalkArgs &a, const double gc[3],
                                           double inv_s, double inv_m, double nq, double no) {
  const double4 c = a.com[j];
  w[0 * STR] = (T)((c.x - gc[0]) * inv_s);
  w[1 * STR] = (T)((c.y - gc[1]) * inv_s);
  w[2 * STR] = (T)((c.z - gc[2]) * inv_s);
  w[3 * STR] = (T)(c.w * inv_m);
  if (ORDER >= 4) {
    if (sizeof(T) == 4) {
      const float4 q0 = a.fq[2 * (int64_t)j], q1 = a.fq[2 * (int64_t)j + 1];
      w[4 * STR] = (T)(7.5f * q0.x); w[5 * STR] = (T)(7.5f * q0.y); w[6 * STR] = (T)(7.5f * q0.z);
      w[7 * STR] = (T)(7.5f * q0.w); w[8 * STR] = (T)(7.5f * q1.x); w[9 * STR] = (T)(7.5f * q1.y);
      w[10 * STR] = (T)(-1.5f * q1.z);
    } else {
      const double *q = a.quad + 6 * (int64_t)j;
      const double q0 = q[0] * nq, q1 = q[1] * nq, q2 = q[2] * nq;
      w[4 * STR] = (T)(7.5 * q0); w[5 * STR] = (T)(7.5 * q1); w[6 * STR] = (T)(7.5 * q2);
      w[7 * STR] = (T)(7.5 * q[3] * nq); w[8 * STR] = (T)(7.5 * q[4] * nq);
      w[9 * STR] = (T)(7.5 * q[5] * nq);
      w[10 * STR] = (T)(-1.5 * (q0 + q1 + q2));
    }
    w[11 * STR] = (T)0;
  }
  if (ORDER >= 8) {
    if (sizeof(T) == 4) {
      const float4 *f = a.fo + 4 * (int64_t)j;
      const float4 o0 = f[0], o1 = f[1], o2 = f[2], o3 = f[3];
      w[12 * STR] = (T)o0.x; w[13 * STR] = (T)o0.y; w[14 * STR] = (T)o0.z; w[15 * STR] = (T)o0.w;
      w[16 * STR] = (T)o1.x; w[17 * STR] = (T)o1.y; w[18 * STR] = (T)o1.z; w[19 * STR] = (T)o1.w;
      w[20 * STR] = (T)o2.x; w[21 * STR] = (T)o2.y; w[22 * STR] = (T)o2.z; w[23 * STR] = (T)o2.w;
      w[11 * STR] = (T)o3.x;
    } else {
      const double *o = a.oct + 14 * (int64_t)j;
      for (int k = 0; k < 10; ++k) w[(12 + k) * STR] = (T)(o[k] * no);
      w[22 * STR] = (T)(o[11] * no);
      w[23 * STR] = (T)(o[12] * no);
      w[11 * STR] = (T)(o[13] * no);
    }
  }
}

// Vector loads of W staged words (float4 / double2).
template <int W>
__device__ __forceinline__ void load_words(const float *p, float (&w)[W]) {
#pragma unroll
  for (int k = 0; k < W; k += 4) {
    const float4 v = *reinterpret_cast<const float4 *>(p + k);
    w[k] = v.x; w[k + 1] = v.y; w[k + 2] = v.z; w[k + 3] = v.w;
  }
}
template <int W>
__device__ __forceinline__ void load_words(const double *p, double (&w)[W]) {
#pragma unroll
  for (int k = 0; k < W; k += 2) {
    const double2 v = *reinterpret_cast<const double2 *>(p + k);
    w[k] = v.x; w[k + 1] = v.y;
  }
}

// Reciprocal square root.  FP32: one approximate hardware instruction
// (rel. error ~2^-22.9) with subnormals flushed: every input is a squared
// distance in units of the root cube side, never subnormal.  FP64: rsqrt().
__device__ __forceinline__ float fast_rsqrt(float x) {
  float r;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ double fast_rsqrt(double x) { return rsqrt(x); }

// (2^-level)^2 = 2^(-2 level), exact, from the exponent bits (level <= 21)
template <typename T> __device__ __forceinline__ T pow2_neg2(int level);
template <> __device__ __forceinline__ float pow2_neg2<float>(int level) {
  return __int_as_float((127 - 2 * level) << 23);
}
template <> __device__ __forceinline__ double pow2_neg2<double>(int level) {
  return __longlong_as_double((long long)(1023 - 2 * level) << 52);
}

// Smallest r^2 of a body pair when there is no softening: a body meets itself
// (d = 0, contribution exactly 0) and exactly coincident bodies contribute 0;
// r^-3 stays finite in T.
template <typename T> __device__ __forceinline__ T r2_floor();
template <> __device__ __forceinline__ float r2_floor<float>() { return 1e-24f; }
template <> __device__ __forceinline__ double r2_floor<double>() { return 1e-200; }

// One body-body term added to (bx, by, bz) (morton_octree.f90:676-686).
template <typename T, bool SOFT>
__device__ __forceinline__ void body_force(T sx, T sy, T sz, T sm, T rx, T ry, T rz, T eps2,
                                           T &bx, T &by, T &bz) {
  const T dx = sx - rx, dy = sy - ry, dz = sz - rz;
  T r2 = fma(dx, dx, fma(dy, dy, fma(dz, dz, eps2)));
  if (!SOFT) r2 = max(r2, r2_floor<T>());
  const T ri = fast_rsqrt(r2);
  const T f = (sm * ri) * (ri * ri);
  bx = fma(f, dx, bx); by = fma(f, dy, by); bz = fma(f, dz, bz);
}

// One cell term added to (bx, by, bz): the reference's grouped-walk formula
// (octree_default.f90:1993-2083) with r^-3 factored out of every term:
//   a += r^-3 [ (M - 1.5 trQ r^-2 + 7.5 dQd r^-4) d - 3 r^-2 Q d + r^3 O(d) ].
// Accepted cells never coincide with a target (the group box lies outside the
// MAC radius), so r^2 > 0.
template <typename T, int ORDER>
__device__ __forceinline__ void cell_force(const T *w, T rx, T ry, T rz, T eps2, T &bx, T &by,
                                           T &bz) {
  const T dx = w[0] - rx, dy = w[1] - ry, dz = w[2] - rz;
  const T r2 = fma(dx, dx, fma(dy, dy, fma(dz, dz, eps2)));
  const T rinv = fast_rsqrt(r2);
  const T r2i = rinv * rinv;
  const T r3i = rinv * r2i;
  if (ORDER < 4) {
    const T f = w[3] * r3i;
    bx = fma(f, dx, bx); by = fma(f, dy, by); bz = fma(f, dz, bz);
    return;
  }
  // w[4..9] = 7.5 Q, w[10] = -1.5 trQ
  const T qx = fma(w[4], dx, fma(w[7], dy, w[8] * dz));
  const T qy = fma(w[7], dx, fma(w[5], dy, w[9] * dz));
  const T qz = fma(w[8], dx, fma(w[9], dy, w[6] * dz));
  const T dqd = fma(dx, qx, fma(dy, qy, dz * qz));          // 7.5 dQd
  const T A = fma(dqd, r2i * r2i, fma(w[10], r2i, w[3]));  // M - 1.5 tr r^-2 + 7.5 dQd r^-4
  const T sA = r3i * A;
  const T t = (T)-0.4 * (r3i * r2i);                        // -3 r^-5 / 7.5
  if (ORDER < 8) {
    bx = fma(sA, dx, fma(t, qx, bx));
    by = fma(sA, dy, fma(t, qy, by));
    bz = fma(sA, dz, fma(t, qz, bz));
    return;
  }
  const T O1 = w[12], O2 = w[13], O3 = w[14], O4 = w[15], O5 = w[16], O6 = w[17], O7 = w[18],
          O8 = w[19], O9 = w[20], O10 = w[21], O12 = w[22], O13 = w[23], O14 = w[11];
  const T s7 = (T)7.5 * r2i * r2i;          // 7.5 r^-4
  const T s5 = (T)-1.5 * r2i;               // -1.5 r^-2
  const T s9 = (T)-17.5 * r2i * r2i * r2i;  // -17.5 r^-6
  const T xx = dx * dx, yy = dy * dy, zz = dz * dz, xy = dx * dy, xz = dx * dz, yz = dy * dz;
  const T oc = s7 * fma(dx, O12, fma(dy, O13, dz * O14));
  T ox = fma(s5, O12, dx * oc), oy = fma(s5, O13, dy * oc), oz = fma(s5, O14, dz * oc);
  ox = fma(s7, fma(xx, O1, fma(yy, O2, zz * O3)) + (T)2 * fma(xy, O4, fma(xz, O7, yz * O10)), ox);
  oy = fma(s7, fma(xx, O4, fma(yy, O5, zz * O6)) + (T)2 * fma(xy, O2, fma(xz, O10, yz * O8)), oy);
  oz = fma(s7, fma(xx, O7, fma(yy, O8, zz * O9)) + (T)2 * fma(xy, O10, fma(xz, O3, yz * O6)), oz);
  T c3 = fma(xx * dx, O1, fma(yy * dy, O5, zz * dz * O9));
  c3 = fma((T)3, fma(xx * dy, O4, fma(xx * dz, O7, xy * dy * O2)), c3);
  c3 = fma((T)3, fma(yy * dz, O8, fma(xz * dz, O3, yz * dz * O6)), c3);
  c3 = fma((T)6 * xy, dz * O10, c3);
  c3 = s9 * c3;
  ox = fma(dx, c3, ox); oy = fma(dy, c3, oy); oz = fma(dz, c3, oz);
  bx = fma(sA, dx, fma(t, qx, fma(r3i, ox, bx)));
  by = fma(sA, dy, fma(t, qy, fma(r3i, oy, by)));
  bz = fma(sA, dz, fma(t, qz, fma(r3i, oz, bz)));
}

// ---- paired FP32 (sm_100 f32x2 instructions) ----
//
// The FP32 walk evaluates two staged entries (cells j and j+1, or bodies) per
// instruction: every operand is a float2 whose halves belong to the two
// entries, and the target's coordinates are the same in both halves.  Each half
// is rounded exactly like the scalar operation it replaces.
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 splat(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 rsqrt2(float2 x) { return make_float2(fast_rsqrt(x.x), fast_rsqrt(x.y)); }

// Two body-body terms; (nrx, nry, nrz) is minus the target's position.
template <bool SOFT>
__device__ __forceinline__ void body_force2(float2 sx, float2 sy, float2 sz, float2 sm, float2 nrx,
                                            float2 nry, float2 nrz, float2 eps2, float2 &bx,
                                            float2 &by, float2 &bz) {
  const float2 dx = add2(sx, nrx), dy = add2(sy, nry), dz = add2(sz, nrz);
  float2 r2 = fma2(dx, dx, fma2(dy, dy, fma2(dz, dz, eps2)));
  if (!SOFT) { r2.x = fmaxf(r2.x, r2_floor<float>()); r2.y = fmaxf(r2.y, r2_floor<float>()); }
  const float2 ri = rsqrt2(r2);
  const float2 f = mul2(mul2(sm, ri), mul2(ri, ri));
  bx = fma2(f, dx, bx); by = fma2(f, dy, by); bz = fma2(f, dz, bz);
}

// Two cell terms, the formula of cell_force; w[k] holds word k of both cells.
template <int ORDER>
__device__ __forceinline__ void cell_force2(const float2 *w, float2 nrx, float2 nry, float2 nrz,
                                            float2 eps2, float2 &bx, float2 &by, float2 &bz) {
  const float2 dx = add2(w[0], nrx), dy = add2(w[1], nry), dz = add2(w[2], nrz);
  const float2 r2 = fma2(dx, dx, fma2(dy, dy, fma2(dz, dz, eps2)));
  const float2 rinv = rsqrt2(r2);
  const float2 r2i = mul2(rinv, rinv);
  const float2 r3i = mul2(rinv, r2i);
  if (ORDER < 4) {
    const float2 f = mul2(w[3], r3i);
    bx = fma2(f, dx, bx); by = fma2(f, dy, by); bz = fma2(f, dz, bz);
    return;
  }
  const float2 qx = fma2(w[4], dx, fma2(w[7], dy, mul2(w[8], dz)));
  const float2 qy = fma2(w[7], dx, fma2(w[5], dy, mul2(w[9], dz)));
  const float2 qz = fma2(w[8], dx, fma2(w[9], dy, mul2(w[6], dz)));
  const float2 dqd = fma2(dx, qx, fma2(dy, qy, mul2(dz, qz)));
  const float2 A = fma2(dqd, mul2(r2i, r2i), fma2(w[10], r2i, w[3]));
  const float2 sA = mul2(r3i, A);
  const float2 t = mul2(splat(-0.4f), mul2(r3i, r2i));
  if (ORDER < 8) {
    bx = fma2(sA, dx, fma2(t, qx, bx));
    by = fma2(sA, dy, fma2(t, qy, by));
    bz = fma2(sA, dz, fma2(t, qz, bz));
    return;
  }
  const float2 O1 = w[12], O2 = w[13], O3 = w[14], O4 = w[15], O5 = w[16], O6 = w[17], O7 = w[18],
               O8 = w[19], O9 = w[20], O10 = w[21], O12 = w[22], O13 = w[23], O14 = w[11];
  const float2 r4i = mul2(r2i, r2i);
  const float2 s7 = mul2(splat(7.5f), r4i);
  const float2 s5 = mul2(splat(-1.5f), r2i);
  const float2 s9 = mul2(mul2(splat(-17.5f), r4i), r2i);
  const float2 xx = mul2(dx, dx), yy = mul2(dy, dy), zz = mul2(dz, dz), xy = mul2(dx, dy),
               xz = mul2(dx, dz), yz = mul2(dy, dz);
  const float2 two = splat(2.0f), three = splat(3.0f);
  const float2 oc = mul2(s7, fma2(dx, O12, fma2(dy, O13, mul2(dz, O14))));
  float2 ox = fma2(s5, O12, mul2(dx, oc)), oy = fma2(s5, O13, mul2(dy, oc)),
         oz = fma2(s5, O14, mul2(dz, oc));
  ox = fma2(s7, fma2(two, fma2(xy, O4, fma2(xz, O7, mul2(yz, O10))),
                     fma2(xx, O1, fma2(yy, O2, mul2(zz, O3)))), ox);
  oy = fma2(s7, fma2(two, fma2(xy, O2, fma2(xz, O10, mul2(yz, O8))),
                     fma2(xx, O4, fma2(yy, O5, mul2(zz, O6)))), oy);
  oz = fma2(s7, fma2(two, fma2(xy, O10, fma2(xz, O3, mul2(yz, O6))),
                     fma2(xx, O7, fma2(yy, O8, mul2(zz, O9)))), oz);
  float2 c3 = fma2(mul2(xx, dx), O1, fma2(mul2(yy, dy), O5, mul2(mul2(zz, dz), O9)));
  c3 = fma2(three, fma2(mul2(xx, dy), O4, fma2(mul2(xx, dz), O7, mul2(mul2(xy, dy), O2))), c3);
  c3 = fma2(three, fma2(mul2(yy, dz), O8, fma2(mul2(xz, dz), O3, mul2(mul2(yz, dz), O6))), c3);
  c3 = fma2(mul2(splat(6.0f), xy), mul2(dz, O10), c3);
  c3 = mul2(s9, c3);
  ox = fma2(dx, c3, ox); oy = fma2(dy, c3, oy); oz = fma2(dz, c3, oz);
  bx = fma2(sA, dx, fma2(t, qx, fma2(r3i, ox, bx)));
  by = fma2(sA, dy, fma2(t, qy, fma2(r3i, oy, by)));
  bz = fma2(sA, dz, fma2(t, qz, fma2(r3i, oz, bz)));
}

// Accepted nodes of at most this many bodies are evaluated body by body
// (6 for the octupole: 12.4 instead of 13.2 ms at N = 2^20; for the
// quadrupole and the monopole no count pays).
template <int ORDER> __host__ __device__ constexpr int bodies_as_cell() { return ORDER >= 8 ? 6 : 1; }

// A staged entry that contributes exactly zero: no mass, no moments, far from
// every target (positions are in root-cube units, |x| <= ~1).
constexpr float kPadPos = 1.0e4f;

struct WalkCounters {
  unsigned long long pp = 0, pc = 0, tests = 0;
  int err = 0;
};

// The tree walk of one group (the box-distance MAC of octree_default.f90
// :1927-1936, optionally with every member's own MAC): accepted nodes are
// queued as cells and the bodies of opened leaves and lone particles as
// bodies; eval_cells(end, k) / eval_bodies(end, k) consume the k queue entries
// that end at position `end`, 32 at a time and the remainders at the end.
// Positions are relative to the group centre gc in units of the root side.
// An accepted node of at most ASB bodies is queued as its bodies: for the
// octupole, whose cell term costs as much as about 8 body terms, that is
// cheaper and exact.
template <typename T, int TPL, int ASB, typename CellsFn, typename BodiesFn>
__device__ __forceinline__ void tree_walk(const WalkArgs &a, int *cellq, int *bodyq,
                                          int32_t *stack, int stack_cap, int gf, int gn, int root,
                                          const double gc[3], double inv_s, const T blo[3],
                                          const T bhi[3], T theta2, T inv_theta2, T diag, T rad,
                                          const T (&rx)[TPL], const T (&ry)[TPL],
                                          const T (&rz)[TPL], WalkCounters &wc,
                                          CellsFn &&eval_cells, BodiesFn &&eval_bodies) {
  const int lane = threadIdx.x & (kWarp - 1);
  const unsigned lt = (1u << lane) - 1u;
  int top = 1, ncell = 0, nbody = 0;
  // a tree visits every node at most once per group: more tests than nodes
  // means a malformed tree, and the walk stops with an error instead of
  // looping
  const int64_t max_tests = (int64_t)a.sc->n_compact + kWarp;
  int64_t group_tests = 0;
  if (root < 0) top = 0;  // a lone body: no tree, no force
  if (lane == 0) stack[0] = root;
  __syncwarp();
  while (top > 0) {
    if (group_tests > max_tests) { wc.err |= kErrIndex; break; }
    const int take = min(top, kWarp);
    const int base = top - take;
    const int node = lane < take ? stack[base + lane] : -1;
    top = base;
    __syncwarp();
    int cls = 0;  // 1 cell, 2 open leaf, 3 open internal
    int4 mt = make_int4(0, 0, 0, 0);
    T dx = (T)0, dy = (T)0, dz = (T)0, size2 = (T)0;
    bool cand = false;
    if (node >= 0) {
      mt = a.meta[node];
      const double4 c = a.com[node];
      dx = (T)((c.x - gc[0]) * inv_s); dy = (T)((c.y - gc[1]) * inv_s); dz = (T)((c.z - gc[2]) * inv_s);
      const T ex = max(max(blo[0] - dx, (T)0), dx - bhi[0]);
      const T ey = max(max(blo[1] - dy, (T)0), dy - bhi[1]);
      const T ez = max(max(blo[2] - dz, (T)0), dz - bhi[2]);
      const T d2 = fma(ex, ex, fma(ey, ey, ez * ez));
      size2 = pow2_neg2<T>(mt.z);
      if (size2 <= theta2 * d2) {
        cls = 1;
      } else {
        cls = (mt.y <= a.leaf_cap || mt.w == 0) ? 2 : 3;
        if (a.mac == 1 && (mt.x + mt.y <= gf || mt.x >= gf + gn)) {
          // holds no member: accept when every member passes its own MAC.
          // Every member is at least |c| - rad from the centre of mass (the
          // sphere bound); otherwise the members are tested one by one below
          // if the nearest of them (at most `diag` beyond the box) may pass.
          const T reach = sqrt(size2 * inv_theta2);
          const T dc = sqrt(fma(dx, dx, fma(dy, dy, dz * dz)));
          if (dc - rad >= reach) {
            cls = 1;
          } else {
            const T r2 = reach - diag;
            cand = r2 <= (T)0 || r2 * r2 <= d2;
          }
        }
      }
    }
    // members' own MAC (morton_octree.f90:701-706: size^2 <= theta^2 d^2 with
    // d from the member to the centre of mass), all members at once
    for (unsigned pend = __ballot_sync(kFull, cand); pend; pend &= pend - 1) {
      const int src = __ffs(pend) - 1;
      const T cx = __shfl_sync(kFull, dx, src), cy = __shfl_sync(kFull, dy, src),
              cz = __shfl_sync(kFull, dz, src), cs2 = __shfl_sync(kFull, size2, src);
      T dmin = (T)INFINITY;
#pragma unroll
      for (int t = 0; t < TPL; ++t) {
        const T ux = cx - rx[t], uy = cy - ry[t], uz = cz - rz[t];
        dmin = min(dmin, fma(ux, ux, fma(uy, uy, uz * uz)));
      }
      dmin = warp_min(dmin);
      if (lane == src && cs2 <= theta2 * dmin) cls = 1;
    }
    if (cls == 1 && mt.y <= ASB) cls = 2;
    wc.tests += take;
    group_tests += take;
    // cells
    const unsigned cm = __ballot_sync(kFull, cls == 1);
    if (cls == 1) cellq[ncell + __popc(cm & lt)] = node;
    ncell += __popc(cm);
    // children of opened internal nodes
    int32_t ch[8];
    int nnc = 0, npc = 0;
    if (cls == 3) {
      const int4 *cp = reinterpret_cast<const int4 *>(a.child + 8 * (int64_t)node);
      const int4 c0 = cp[0], c1 = cp[1];
      ch[0] = c0.x; ch[1] = c0.y; ch[2] = c0.z; ch[3] = c0.w;
      ch[4] = c1.x; ch[5] = c1.y; ch[6] = c1.z; ch[7] = c1.w;
#pragma unroll
      for (int c = 0; c < 8; ++c)
        if (c < mt.w) { if (ch[c] >= 0) ++nnc; else ++npc; }
    }
    int tot;
    const int soff = warp_excl_scan(nnc, lane, tot);
    if (top + tot > stack_cap) {
      // capacity exceeded: the group's result is incomplete and flagged;
      // the host repeats the walk with a larger stack
      wc.err |= kErrStackOverflow;
    } else {
      if (cls == 3) {
        int k = top + soff;
#pragma unroll
        for (int c = 0; c < 8; ++c)
          if (c < mt.w && ch[c] >= 0) stack[k++] = ch[c];
      }
      top += tot;
    }
    // bodies: lone-particle children (<= 8, one pass) and leaf ranges
    int rf = 0, rn = 0;
    if (cls == 2) { rf = mt.x; rn = mt.y; }
    bool first_pass = true;
    // nothing to queue on any lane (the common case): no scan
    for (bool any = __ballot_sync(kFull, rn > 0 || (cls == 3 && npc > 0)) != 0u; any;
         any = __ballot_sync(kFull, rn > 0) != 0u) {
      int give;
      if (first_pass && cls == 3) give = npc;
      else give = min(rn, kBodyPerLane);
      int btot;
      const int boff = warp_excl_scan(give, lane, btot);
      if (btot == 0) break;
      if (first_pass && cls == 3) {
        int k = nbody + boff;
#pragma unroll
        for (int c = 0; c < 8; ++c)
          if (c < mt.w && ch[c] < 0) bodyq[k++] = ~ch[c];
      } else {
        for (int k = 0; k < give; ++k) bodyq[nbody + boff + k] = rf + k;
        rf += give; rn -= give;
      }
      first_pass = false;
      nbody += btot;
      __syncwarp();
      while (nbody >= kWarp) { eval_bodies(nbody, kWarp); nbody -= kWarp; }
    }
    __syncwarp();
    while (ncell >= kWarp) { eval_cells(ncell, kWarp); ncell -= kWarp; }
    __syncwarp();
  }
  if (ncell > 0) eval_cells(ncell, ncell);
  if (nbody > 0) eval_bodies(nbody, nbody);
}

// One group: TPL targets per lane (the group has <= 32 * TPL bodies).
template <typename T, int ORDER, int TPL, bool SOFT>
__device__ __forceinline__ void walk_group(const WalkArgs &a, WarpSmem<T, ORDER> &S,
                                           int32_t *stack, int stack_cap, int gf, int gn,
                                           const SysScalars &ss, T theta2, WalkCounters &wc) {
  const double inv_s = 1.0 / ss.ssa, inv_m = 1.0 / ss.mass;
  const double nq = inv_m * inv_s * inv_s, no = nq * inv_s;
  const T eps2 = (T)(a.eps2 * inv_s * inv_s);
  const int root = ss.root;
  constexpr int W = StageWords<ORDER>::value;
  constexpr bool kKahan = sizeof(T) == 4;
  const int lane = threadIdx.x & (kWarp - 1);

  double px[TPL], py[TPL], pz[TPL];
  bool valid[TPL];
#pragma unroll
  for (int t = 0; t < TPL; ++t) {
    const int k = lane + kWarp * t;
    valid[t] = k < gn;
    const double4 p = a.spos[gf + (valid[t] ? k : 0)];
    px[t] = p.x; py[t] = p.y; pz[t] = p.z;
  }
  double lo[3] = {px[0], py[0], pz[0]}, hi[3] = {px[0], py[0], pz[0]};
#pragma unroll
  for (int t = 1; t < TPL; ++t) {
    lo[0] = fmin(lo[0], px[t]); hi[0] = fmax(hi[0], px[t]);
    lo[1] = fmin(lo[1], py[t]); hi[1] = fmax(hi[1], py[t]);
    lo[2] = fmin(lo[2], pz[t]); hi[2] = fmax(hi[2], pz[t]);
  }
  double gc[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) gc[k] = 0.5 * (warp_min(lo[k]) + warp_max(hi[k]));
  T rx[TPL], ry[TPL], rz[TPL];
  T ax[TPL], ay[TPL], az[TPL], cx[TPL], cy[TPL], cz[TPL];
  T blo[3], bhi[3];
#pragma unroll
  for (int t = 0; t < TPL; ++t) {
    rx[t] = (T)((px[t] - gc[0]) * inv_s);
    ry[t] = (T)((py[t] - gc[1]) * inv_s);
    rz[t] = (T)((pz[t] - gc[2]) * inv_s);
    ax[t] = ay[t] = az[t] = cx[t] = cy[t] = cz[t] = (T)0;
    if (t == 0) { blo[0] = bhi[0] = rx[0]; blo[1] = bhi[1] = ry[0]; blo[2] = bhi[2] = rz[0]; }
    else {
      blo[0] = min(blo[0], rx[t]); bhi[0] = max(bhi[0], rx[t]);
      blo[1] = min(blo[1], ry[t]); bhi[1] = max(bhi[1], ry[t]);
      blo[2] = min(blo[2], rz[t]); bhi[2] = max(bhi[2], rz[t]);
    }
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) { blo[k] = warp_min(blo[k]); bhi[k] = warp_max(bhi[k]); }
  // every member lies within `diag` of every point of the box
  const T diag = sqrt((bhi[0] - blo[0]) * (bhi[0] - blo[0]) + (bhi[1] - blo[1]) * (bhi[1] - blo[1]) +
                      (bhi[2] - blo[2]) * (bhi[2] - blo[2]));
  const T inv_theta2 = theta2 > (T)0 ? (T)1 / theta2 : (T)INFINITY;
  // radius of the members' sphere about the group centre
  T rad2 = (T)0;
#pragma unroll
  for (int t = 0; t < TPL; ++t) rad2 = max(rad2, fma(rx[t], rx[t], fma(ry[t], ry[t], rz[t] * rz[t])));
  const T rad = sqrt(warp_max(rad2));

  auto accumulate = [&](const T (&bx)[TPL], const T (&by)[TPL], const T (&bz)[TPL]) {
#pragma unroll
    for (int t = 0; t < TPL; ++t) {
      if (kKahan) {
        kahan_add(ax[t], cx[t], bx[t]); kahan_add(ay[t], cy[t], by[t]); kahan_add(az[t], cz[t], bz[t]);
      } else {
        ax[t] += bx[t]; ay[t] += by[t]; az[t] += bz[t];
      }
    }
  };
  // FP32: paired evaluation; target coordinates negated and duplicated once
  constexpr bool kPaired = sizeof(T) == 4;
  float2 nrx[TPL], nry[TPL], nrz[TPL];
#pragma unroll
  for (int t = 0; t < TPL; ++t) {
    nrx[t] = splat(-(float)rx[t]); nry[t] = splat(-(float)ry[t]); nrz[t] = splat(-(float)rz[t]);
  }
  const float2 eps2p = splat((float)eps2);
  // evaluate the nb queue entries ending at position `end`
  auto eval_bodies = [&](int end, int nb) {
    if constexpr (kPaired) {
      // stage: body pair i at [8i, 8i + 8) as (x, x', y, y', z, z', m, m'); an
      // odd count is padded with a massless far body
      float *w = reinterpret_cast<float *>(S.stage) + (lane >> 1) * 8 + (lane & 1);
      if (lane < nb) {
        const int p = S.bodyq[end - nb + lane];
        const double4 s = a.spos[p];
        w[0] = (float)((s.x - gc[0]) * inv_s);
        w[2] = (float)((s.y - gc[1]) * inv_s);
        w[4] = (float)((s.z - gc[2]) * inv_s);
        w[6] = (float)(s.w * inv_m);
      } else if (lane == nb && (nb & 1)) {
        w[0] = w[2] = w[4] = kPadPos;
        w[6] = 0.0f;
      }
      __syncwarp();
      float2 bx[TPL], by[TPL], bz[TPL];
#pragma unroll
      for (int t = 0; t < TPL; ++t) bx[t] = by[t] = bz[t] = make_float2(0.0f, 0.0f);
      const int np = (nb + 1) >> 1;
      const float4 *st = reinterpret_cast<const float4 *>(S.stage);
      for (int j = 0; j < np; ++j) {
        const float4 u = st[2 * j], v = st[2 * j + 1];
        const float2 sx = make_float2(u.x, u.y), sy = make_float2(u.z, u.w);
        const float2 sz = make_float2(v.x, v.y), sm = make_float2(v.z, v.w);
#pragma unroll
        for (int t = 0; t < TPL; ++t)
          body_force2<SOFT>(sx, sy, sz, sm, nrx[t], nry[t], nrz[t], eps2p, bx[t], by[t], bz[t]);
      }
      T sx[TPL], sy[TPL], sz[TPL];
#pragma unroll
      for (int t = 0; t < TPL; ++t) {
        sx[t] = bx[t].x + bx[t].y; sy[t] = by[t].x + by[t].y; sz[t] = bz[t].x + bz[t].y;
      }
      accumulate(sx, sy, sz);
    } else {
      if (lane < nb) {
        const int p = S.bodyq[end - nb + lane];
        const double4 s = a.spos[p];
        T *w = S.stage + lane * 4;
        w[0] = (T)((s.x - gc[0]) * inv_s);
        w[1] = (T)((s.y - gc[1]) * inv_s);
        w[2] = (T)((s.z - gc[2]) * inv_s);
        w[3] = (T)(s.w * inv_m);
      }
      __syncwarp();
      T bx[TPL], by[TPL], bz[TPL];
#pragma unroll
      for (int t = 0; t < TPL; ++t) bx[t] = by[t] = bz[t] = (T)0;
#pragma unroll 2
      for (int j = 0; j < nb; ++j) {
        T w[4];
        load_words<4>(S.stage + j * 4, w);
#pragma unroll
        for (int t = 0; t < TPL; ++t)
          body_force<T, SOFT>(w[0], w[1], w[2], w[3], rx[t], ry[t], rz[t], eps2, bx[t], by[t], bz[t]);
      }
      accumulate(bx, by, bz);
    }
    wc.pp += (unsigned long long)nb * gn;
    __syncwarp();
  };
  auto eval_cells = [&](int end, int nc) {
    if constexpr (kPaired) {
      // stage: cell pair i at [2Wi, 2W(i + 1)), word k of both cells at 2k, 2k + 1;
      // an odd count is padded with an empty far cell
      float *w = reinterpret_cast<float *>(S.stage) + (lane >> 1) * 2 * W + (lane & 1);
      if (lane < nc) {
        stage_cell<float, ORDER, 2>(w, S.cellq[end - nc + lane], a, gc, inv_s, inv_m, nq, no);
      } else if (lane == nc && (nc & 1)) {
#pragma unroll
        for (int k = 3; k < W; ++k) w[2 * k] = 0.0f;
        w[0] = w[2] = w[4] = kPadPos;
      }
      __syncwarp();
      float2 bx[TPL], by[TPL], bz[TPL];
#pragma unroll
      for (int t = 0; t < TPL; ++t) bx[t] = by[t] = bz[t] = make_float2(0.0f, 0.0f);
      const int np = (nc + 1) >> 1;
#pragma unroll 2
      for (int j = 0; j < np; ++j) {
        const float4 *st = reinterpret_cast<const float4 *>(S.stage) + j * (W / 2);
        float2 cw[W];
#pragma unroll
        for (int k = 0; k < W / 2; ++k) {
          const float4 v = st[k];
          cw[2 * k] = make_float2(v.x, v.y);
          cw[2 * k + 1] = make_float2(v.z, v.w);
        }
#pragma unroll
        for (int t = 0; t < TPL; ++t)
          cell_force2<ORDER>(cw, nrx[t], nry[t], nrz[t], eps2p, bx[t], by[t], bz[t]);
      }
      T sx[TPL], sy[TPL], sz[TPL];
#pragma unroll
      for (int t = 0; t < TPL; ++t) {
        sx[t] = bx[t].x + bx[t].y; sy[t] = by[t].x + by[t].y; sz[t] = bz[t].x + bz[t].y;
      }
      accumulate(sx, sy, sz);
    } else {
      if (lane < nc)
        stage_cell<T, ORDER>(S.stage + lane * W, S.cellq[end - nc + lane], a, gc, inv_s, inv_m, nq, no);
      __syncwarp();
      T bx[TPL], by[TPL], bz[TPL];
#pragma unroll
      for (int t = 0; t < TPL; ++t) bx[t] = by[t] = bz[t] = (T)0;
#pragma unroll 2
      for (int j = 0; j < nc; ++j) {
        T w[W];
        load_words<W>(S.stage + j * W, w);
#pragma unroll
        for (int t = 0; t < TPL; ++t) cell_force<T, ORDER>(w, rx[t], ry[t], rz[t], eps2, bx[t], by[t], bz[t]);
      }
      accumulate(bx, by, bz);
    }
    wc.pc += (unsigned long long)nc * gn;
    __syncwarp();
  };

  tree_walk<T, TPL, bodies_as_cell<ORDER>()>(a, S.cellq, S.bodyq, stack, stack_cap, gf, gn, root, gc, inv_s, blo, bhi,
                    theta2, inv_theta2, diag, rad, rx, ry, rz, wc, eval_cells, eval_bodies);

  // forces in the original order; every system's result is an (n_s, 3)
  // Fortran-ordered block at 3 * off_s
  const double scale = a.G * ss.mass * inv_s * inv_s;
  double *out = a.out + 3 * ss.off;
  const int64_t ns = ss.n;
#pragma unroll
  for (int t = 0; t < TPL; ++t) {
    if (!valid[t]) continue;
    const int i = gf + lane + kWarp * t;
    const int64_t p = a.perm[i] - ss.off;
    double fxs = (double)ax[t], fys = (double)ay[t], fzs = (double)az[t];
    if (kKahan) { fxs -= (double)cx[t]; fys -= (double)cy[t]; fzs -= (double)cz[t]; }
    double sc = scale;
    if (a.out_kind == 0) sc *= a.spos[i].w;
    out[p] = fxs * sc;
    out[ns + p] = fys * sc;
    out[2 * ns + p] = fzs * sc;
  }
}

// Persistent warps, one per block, take groups from a global cursor until
// none is left; block b uses stack slot b.  With 64-body groups a group of
// <= 32 bodies runs the one-target-per-lane path.
template <typename T, int ORDER, int MAXTPL, bool SOFT>
__global__ void __launch_bounds__(kWarp, walk_min_blocks<T, ORDER>())
group_walk_kernel(WalkArgs a) {
  __shared__ WarpSmem<T, ORDER> S;
  const int lane = threadIdx.x;
  int32_t *stack = a.stack + (int64_t)blockIdx.x * a.stack_cap;
  const int stack_cap = (int)a.stack_cap;
  const int ngroups = a.g_end >= 0 ? min(a.g_end, a.sc->n_groups) : a.sc->n_groups;
  const T theta2 = (T)a.theta2;
  WalkCounters wc;
  for (;;) {
    int g = 0;
    if (lane == 0) g = a.g_begin + atomicAdd(a.cursor, 1);
    g = __shfl_sync(kFull, g, 0);
    if (g >= ngroups) break;
    const int gf = a.g_first[g];
    const int gn = a.g_first[g + 1] - gf;
    const SysScalars &ss = a.ss[a.sys_of[gf]];
    if (MAXTPL == 2 && gn > kWarp)
      walk_group<T, ORDER, 2, SOFT>(a, S, stack, stack_cap, gf, gn, ss, theta2, wc);
    else
      walk_group<T, ORDER, 1, SOFT>(a, S, stack, stack_cap, gf, gn, ss, theta2, wc);
  }
  if (wc.err && lane == 0) atomicOr(&a.sc->err, wc.err);
  if (a.count_stats && lane == 0) {
    atomicAdd(&a.stats[0], wc.pp);
    atomicAdd(&a.stats[1], wc.pc);
    atomicAdd(&a.stats[3], wc.tests);
  }
}

// ---- warp-specialised FP32 group walk (pipeline = 1) ----
//
// A block holds kTeams teams of one producer warp and one consumer warp.
// The producer takes groups from the global cursor, walks the tree exactly as
// the one-warp walk does and stages every batch of 32 cells or bodies into a
// ring of kRing shared-memory slots; its consumer evaluates the batches and
// writes the forces.  Every target sees the batches of the one-warp walk in
// the same order with the same arithmetic, so the results are the same bit
// for bit; the tree walk of one group overlaps the evaluation of another.
// Producers (warpgroup 0) hand registers to the consumers (warpgroup 1) with
// setmaxnreg, so that more teams fit on an SM.  Each slot has a "full"
// mbarrier (32 arrivals: the producer's lanes) and an "empty" one (32
// arrivals: the consumer's lanes).  Every wait is bounded: a wait that lasts
// more than about 2 s, or sees the block's abort flag, gives up, sets the flag
// and reports an error; every warp of the block then leaves its loop.

constexpr int kTeams = 4;
constexpr int kRing = 4;
constexpr long long kWaitCycles = 4000000000LL;
constexpr int kRingStart = 1, kRingCells = 2, kRingBodies = 3, kRingEnd = 4, kRingQuit = 5;

template <int ORDER>
struct __align__(16) RingSlot {
  int kind, count, g, unused;
  double gc[3];
  double unused2;
  float stage[kWarp * StageWords<ORDER>::value];
};

template <int ORDER>
struct __align__(16) PipeSmem {
  unsigned long long full[kTeams][kRing];
  unsigned long long empty[kTeams][kRing];
  int abort_flag;
  int cellq[kTeams][kCellQ];
  int bodyq[kTeams][kBodyQ];
  RingSlot<ORDER> ring[kTeams][kRing];
};

__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long *b, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned long long *b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
}
__device__ __forceinline__ bool mbar_test(unsigned long long *b, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// The whole warp waits for the phase of parity `parity` of barrier b to
// complete; false when the block was aborted or the wait lasted more than
// `limit` cycles (which aborts the block).
__device__ __forceinline__ bool mbar_wait_warp(unsigned long long *b, unsigned parity,
                                               volatile int *abort_flag,
                                               long long limit = kWaitCycles) {
  const long long t0 = clock64();
  for (;;) {
    const bool ok = mbar_test(b, parity);
    if (__all_sync(kFull, ok)) return true;
    int stop = 0;
    if ((threadIdx.x & (kWarp - 1)) == 0) {
      if (*abort_flag) stop = 1;
      else if (clock64() - t0 > limit) { *abort_flag = 1; stop = 1; }
    }
    if (__shfl_sync(kFull, stop, 0)) return false;
  }
}

// Producer side of one group: the target set-up and tree walk of walk_group,
// with every batch staged into the ring.  `alive` turns false (for the rest
// of the kernel) when a wait gave up.
template <int ORDER, int TPL, bool SOFT>
__device__ __forceinline__ void produce_group(const WalkArgs &a, PipeSmem<ORDER> &P, int team,
                                              int &it, bool &alive, volatile int *abort_flag,
                                              int32_t *stack, int stack_cap, int g, int gf,
                                              int gn, const SysScalars &ss, float theta2,
                                              WalkCounters &wc) {
  using T = float;
  const double inv_s = 1.0 / ss.ssa, inv_m = 1.0 / ss.mass;
  const double nq = inv_m * inv_s * inv_s, no = nq * inv_s;
  constexpr int W = StageWords<ORDER>::value;
  const int lane = threadIdx.x & (kWarp - 1);
  double px[TPL], py[TPL], pz[TPL];
#pragma unroll
  for (int t = 0; t < TPL; ++t) {
    const int k = lane + kWarp * t;
    const double4 p = a.spos[gf + (k < gn ? k : 0)];
    px[t] = p.x; py[t] = p.y; pz[t] = p.z;
  }
  double lo[3] = {px[0], py[0], pz[0]}, hi[3] = {px[0], py[0], pz[0]};
#pragma unroll
  for (int t = 1; t < TPL; ++t) {
    lo[0] = fmin(lo[0], px[t]); hi[0] = fmax(hi[0], px[t]);
    lo[1] = fmin(lo[1], py[t]); hi[1] = fmax(hi[1], py[t]);
    lo[2] = fmin(lo[2], pz[t]); hi[2] = fmax(hi[2], pz[t]);
  }
  double gc[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) gc[k] = 0.5 * (warp_min(lo[k]) + warp_max(hi[k]));
  T rx[TPL], ry[TPL], rz[TPL], blo[3], bhi[3];
#pragma unroll
  for (int t = 0; t < TPL; ++t) {
    rx[t] = (T)((px[t] - gc[0]) * inv_s);
    ry[t] = (T)((py[t] - gc[1]) * inv_s);
    rz[t] = (T)((pz[t] - gc[2]) * inv_s);
    if (t == 0) { blo[0] = bhi[0] = rx[0]; blo[1] = bhi[1] = ry[0]; blo[2] = bhi[2] = rz[0]; }
    else {
      blo[0] = min(blo[0], rx[t]); bhi[0] = max(bhi[0], rx[t]);
      blo[1] = min(blo[1], ry[t]); bhi[1] = max(bhi[1], ry[t]);
      blo[2] = min(blo[2], rz[t]); bhi[2] = max(bhi[2], rz[t]);
    }
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) { blo[k] = warp_min(blo[k]); bhi[k] = warp_max(bhi[k]); }
  const T diag = sqrt((bhi[0] - blo[0]) * (bhi[0] - blo[0]) + (bhi[1] - blo[1]) * (bhi[1] - blo[1]) +
                      (bhi[2] - blo[2]) * (bhi[2] - blo[2]));
  const T inv_theta2 = theta2 > (T)0 ? (T)1 / theta2 : (T)INFINITY;
  T rad2 = (T)0;
#pragma unroll
  for (int t = 0; t < TPL; ++t) rad2 = max(rad2, fma(rx[t], rx[t], fma(ry[t], ry[t], rz[t] * rz[t])));
  const T rad = sqrt(warp_max(rad2));

  // the next slot, once its consumer has released it
  auto acquire = [&]() -> RingSlot<ORDER> * {
    const int slot = it % kRing;
    const unsigned round = (unsigned)(it / kRing);
    if (alive && round > 0 && !mbar_wait_warp(&P.empty[team][slot], (round - 1) & 1u, abort_flag))
      alive = false;
    return &P.ring[team][slot];
  };
  auto publish = [&]() {
    __syncwarp();
    mbar_arrive(&P.full[team][it % kRing]);
    ++it;
  };
  RingSlot<ORDER> *R = acquire();
  if (alive) {
    if (lane == 0) {
      R->kind = kRingStart; R->g = g; R->count = gn;
      R->gc[0] = gc[0]; R->gc[1] = gc[1]; R->gc[2] = gc[2];
    }
    publish();
  }
  // the stage layouts of walk_group's paired evaluation
  auto emit_cells = [&](int end, int nc) {
    RingSlot<ORDER> *Q = acquire();
    if (!alive) return;
    float *w = Q->stage + (lane >> 1) * 2 * W + (lane & 1);
    if (lane < nc) {
      stage_cell<float, ORDER, 2>(w, P.cellq[team][end - nc + lane], a, gc, inv_s, inv_m, nq, no);
    } else if (lane == nc && (nc & 1)) {
#pragma unroll
      for (int k = 3; k < W; ++k) w[2 * k] = 0.0f;
      w[0] = w[2] = w[4] = kPadPos;
    }
    if (lane == 0) { Q->kind = kRingCells; Q->count = nc; }
    wc.pc += (unsigned long long)nc * gn;
    publish();
  };
  auto emit_bodies = [&](int end, int nb) {
    RingSlot<ORDER> *Q = acquire();
    if (!alive) return;
    float *w = Q->stage + (lane >> 1) * 8 + (lane & 1);
    if (lane < nb) {
      const int p = P.bodyq[team][end - nb + lane];
      const double4 sp = a.spos[p];
      w[0] = (float)((sp.x - gc[0]) * inv_s);
      w[2] = (float)((sp.y - gc[1]) * inv_s);
      w[4] = (float)((sp.z - gc[2]) * inv_s);
      w[6] = (float)(sp.w * inv_m);
    } else if (lane == nb && (nb & 1)) {
      w[0] = w[2] = w[4] = kPadPos;
      w[6] = 0.0f;
    }
    if (lane == 0) { Q->kind = kRingBodies; Q->count = nb; }
    wc.pp += (unsigned long long)nb * gn;
    publish();
  };
  tree_walk<T, TPL, bodies_as_cell<ORDER>()>(a, P.cellq[team], P.bodyq[team], stack, stack_cap, gf, gn, ss.root, gc, inv_s,
                    blo, bhi, theta2, inv_theta2, diag, rad, rx, ry, rz, wc, emit_cells,
                    emit_bodies);
  R = acquire();
  if (alive) {
    if (lane == 0) R->kind = kRingEnd;
    publish();
  }
}

// Consumer side of one group (its start slot already read and released):
// evaluates batches until the group's end slot, then writes the forces as
// walk_group does; false when a wait gave up.
template <int ORDER, int TPL, bool SOFT>
__device__ __forceinline__ bool consume_group(const WalkArgs &a, PipeSmem<ORDER> &P, int team,
                                              int &it, volatile int *abort_flag, int gf, int gn,
                                              const double gc[3], const SysScalars &ss) {
  using T = float;
  constexpr int W = StageWords<ORDER>::value;
  const int lane = threadIdx.x & (kWarp - 1);
  const double inv_s = 1.0 / ss.ssa;
  const T eps2 = (T)(a.eps2 * inv_s * inv_s);
  const float2 eps2p = splat(eps2);
  bool valid[TPL];
  float2 nrx[TPL], nry[TPL], nrz[TPL];
  T ax[TPL], ay[TPL], az[TPL], cx[TPL], cy[TPL], cz[TPL];
#pragma unroll
  for (int t = 0; t < TPL; ++t) {
    const int k = lane + kWarp * t;
    valid[t] = k < gn;
    const double4 p = a.spos[gf + (valid[t] ? k : 0)];
    nrx[t] = splat(-(T)((p.x - gc[0]) * inv_s));
    nry[t] = splat(-(T)((p.y - gc[1]) * inv_s));
    nrz[t] = splat(-(T)((p.z - gc[2]) * inv_s));
    ax[t] = ay[t] = az[t] = cx[t] = cy[t] = cz[t] = (T)0;
  }
  for (;;) {
    const int slot = it % kRing;
    const unsigned round = (unsigned)(it / kRing);
    if (!mbar_wait_warp(&P.full[team][slot], round & 1u, abort_flag)) return false;
    const RingSlot<ORDER> &R = P.ring[team][slot];
    const int kind = R.kind, cnt = R.count;
    if (kind == kRingCells) {
      float2 bx[TPL], by[TPL], bz[TPL];
#pragma unroll
      for (int t = 0; t < TPL; ++t) bx[t] = by[t] = bz[t] = make_float2(0.0f, 0.0f);
      const int np = (cnt + 1) >> 1;
#pragma unroll 2
      for (int j = 0; j < np; ++j) {
        const float4 *st = reinterpret_cast<const float4 *>(R.stage) + j * (W / 2);
        float2 cw[W];
#pragma unroll
        for (int k = 0; k < W / 2; ++k) {
          const float4 v = st[k];
          cw[2 * k] = make_float2(v.x, v.y);
          cw[2 * k + 1] = make_float2(v.z, v.w);
        }
#pragma unroll
        for (int t = 0; t < TPL; ++t)
          cell_force2<ORDER>(cw, nrx[t], nry[t], nrz[t], eps2p, bx[t], by[t], bz[t]);
      }
#pragma unroll
      for (int t = 0; t < TPL; ++t) {
        kahan_add(ax[t], cx[t], bx[t].x + bx[t].y);
        kahan_add(ay[t], cy[t], by[t].x + by[t].y);
        kahan_add(az[t], cz[t], bz[t].x + bz[t].y);
      }
    } else if (kind == kRingBodies) {
      float2 bx[TPL], by[TPL], bz[TPL];
#pragma unroll
      for (int t = 0; t < TPL; ++t) bx[t] = by[t] = bz[t] = make_float2(0.0f, 0.0f);
      const int np = (cnt + 1) >> 1;
      const float4 *st = reinterpret_cast<const float4 *>(R.stage);
      for (int j = 0; j < np; ++j) {
        const float4 u = st[2 * j], v = st[2 * j + 1];
        const float2 sx = make_float2(u.x, u.y), sy = make_float2(u.z, u.w);
        const float2 sz = make_float2(v.x, v.y), sm = make_float2(v.z, v.w);
#pragma unroll
        for (int t = 0; t < TPL; ++t)
          body_force2<SOFT>(sx, sy, sz, sm, nrx[t], nry[t], nrz[t], eps2p, bx[t], by[t], bz[t]);
      }
#pragma unroll
      for (int t = 0; t < TPL; ++t) {
        kahan_add(ax[t], cx[t], bx[t].x + bx[t].y);
        kahan_add(ay[t], cy[t], by[t].x + by[t].y);
        kahan_add(az[t], cz[t], bz[t].x + bz[t].y);
      }
    }
    __syncwarp();
    mbar_arrive(&P.empty[team][slot]);
    ++it;
    if (kind == kRingEnd) break;
  }
  const double scale = a.G * ss.mass * inv_s * inv_s;
  double *out = a.out + 3 * ss.off;
  const int64_t ns = ss.n;
#pragma unroll
  for (int t = 0; t < TPL; ++t) {
    if (!valid[t]) continue;
    const int i = gf + lane + kWarp * t;
    const int64_t p = a.perm[i] - ss.off;
    double fxs = (double)ax[t], fys = (double)ay[t], fzs = (double)az[t];
    fxs -= (double)cx[t]; fys -= (double)cy[t]; fzs -= (double)cz[t];
    double sc = scale;
    if (a.out_kind == 0) sc *= a.spos[i].w;
    out[p] = fxs * sc;
    out[ns + p] = fys * sc;
    out[2 * ns + p] = fzs * sc;
  }
  return true;
}

// PipeRegs<ORDER>::blocks blocks of 2 kTeams warps per SM.  At launch every
// thread holds `regs` registers (the most that `blocks` blocks allow); the
// producer warpgroup then gives registers up to the consumer warpgroup:
// producer + consumer = 2 regs, so the consumers' request is always covered by
// the block's own registers (the host checks the launch count first).  The
// quadrupole consumer runs without spills at 96, the octupole one needs more.
constexpr int kPipeThreads = 2 * kTeams * kWarp;
static_assert(kTeams == 4, "one warpgroup of producers, one of consumers");
template <int ORDER> struct PipeRegs {
  static constexpr int blocks = ORDER >= 8 ? 2 : 3;
  static constexpr int regs = ORDER >= 8 ? 128 : 80;
  static constexpr int producer = ORDER >= 8 ? 96 : 64;
  static constexpr int consumer = 2 * regs - producer;
  static_assert(regs * kPipeThreads * blocks <= 65536, "register file");
  static_assert(regs % 8 == 0 && producer % 8 == 0 && consumer <= 256, "setmaxnreg counts");
};

template <int ORDER, int MAXTPL, bool SOFT>
__global__ void __launch_bounds__(kPipeThreads, PipeRegs<ORDER>::blocks)
pipe_walk_kernel(WalkArgs a) {
  extern __shared__ __align__(16) unsigned char pipe_smem_raw[];
  PipeSmem<ORDER> &P = *reinterpret_cast<PipeSmem<ORDER> *>(pipe_smem_raw);
  const int warp = threadIdx.x / kWarp, lane = threadIdx.x & (kWarp - 1);
  if (threadIdx.x == 0) {
    for (int q = 0; q < kTeams; ++q)
      for (int r = 0; r < kRing; ++r) {
        mbar_init(&P.full[q][r], kWarp);
        mbar_init(&P.empty[q][r], kWarp);
      }
    P.abort_flag = 0;
  }
  __syncthreads();
  volatile int *abort_flag = &P.abort_flag;
  const int ngroups = a.g_end >= 0 ? min(a.g_end, a.sc->n_groups) : a.sc->n_groups;
  int it = 0;
  if (warp < kTeams) {
    asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(PipeRegs<ORDER>::producer));
    const int team = warp;
    int32_t *stack = a.stack + ((int64_t)blockIdx.x * kTeams + team) * a.stack_cap;
    const int stack_cap = (int)a.stack_cap;
    const float theta2 = (float)a.theta2;
    WalkCounters wc;
    bool alive = true;
    for (;;) {
      int g = 0;
      if (lane == 0) g = a.g_begin + atomicAdd(a.cursor, 1);
      g = __shfl_sync(kFull, g, 0);
      if (g >= ngroups) break;
      const int gf = a.g_first[g];
      const int gn = a.g_first[g + 1] - gf;
      const SysScalars &ss = a.ss[a.sys_of[gf]];
      if (MAXTPL == 2 && gn > kWarp)
        produce_group<ORDER, 2, SOFT>(a, P, team, it, alive, abort_flag, stack, stack_cap, g, gf,
                                      gn, ss, theta2, wc);
      else
        produce_group<ORDER, 1, SOFT>(a, P, team, it, alive, abort_flag, stack, stack_cap, g, gf,
                                      gn, ss, theta2, wc);
      if (!alive) break;
    }
    if (alive) {  // tell the consumer there is nothing more
      const int slot = it % kRing;
      const unsigned round = (unsigned)(it / kRing);
      if (round == 0 || mbar_wait_warp(&P.empty[team][slot], (round - 1) & 1u, abort_flag)) {
        if (lane == 0) P.ring[team][slot].kind = kRingQuit;
        __syncwarp();
        mbar_arrive(&P.full[team][slot]);
      }
    }
    if (lane == 0) {
      if (wc.err) atomicOr(&a.sc->err, wc.err);
      if (!alive) atomicOr(&a.sc->err, kErrTimeout);
      if (a.count_stats) {
        atomicAdd(&a.stats[0], wc.pp);
        atomicAdd(&a.stats[1], wc.pc);
        atomicAdd(&a.stats[3], wc.tests);
      }
    }
  } else {
    asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" ::"n"(PipeRegs<ORDER>::consumer));
    const int team = warp - kTeams;
    for (;;) {
      const int slot = it % kRing;
      const unsigned round = (unsigned)(it / kRing);
      if (!mbar_wait_warp(&P.full[team][slot], round & 1u, abort_flag)) {
        if (lane == 0) atomicOr(&a.sc->err, kErrTimeout);
        break;
      }
      const RingSlot<ORDER> &R = P.ring[team][slot];
      const int kind = R.kind, g = R.g, gn = R.count;
      const double gc[3] = {R.gc[0], R.gc[1], R.gc[2]};
      __syncwarp();
      mbar_arrive(&P.empty[team][slot]);
      ++it;
      if (kind != kRingStart) break;  // the producer has no more groups
      const int gf = a.g_first[g];
      const SysScalars &ss = a.ss[a.sys_of[gf]];
      bool ok;
      if (MAXTPL == 2 && gn > kWarp)
        ok = consume_group<ORDER, 2, SOFT>(a, P, team, it, abort_flag, gf, gn, gc, ss);
      else
        ok = consume_group<ORDER, 1, SOFT>(a, P, team, it, abort_flag, gf, gn, gc, ss);
      if (!ok) {
        if (lane == 0) atomicOr(&a.sc->err, kErrTimeout);
        break;
      }
    }
  }
}

// Check of the bounded waits above on one block of two warps.  Warp 0 arrives
// at barrier 2 (a phase that completes), waits until warp 1 has seen it
// complete, then waits on barrier 0, at which nothing ever arrives, for
// `limit` cycles.  Warp 1 waits on barrier 2, acknowledges on barrier 1, then
// waits on barrier 0 with the walk's full limit: it must be released by the
// abort flag that warp 0 sets when it gives up.  out: [0] warp 0's result on
// barrier 0, [1] warp 1's result on barrier 2, [2] warp 1's result on barrier
// 0, [3] the cycles warp 1 waited there, [4] the abort flag at the end.
__global__ void __launch_bounds__(2 * kWarp) wait_probe_kernel(long long limit, long long *out) {
  __shared__ __align__(8) unsigned long long bar[3];
  __shared__ int abort_flag;
  const int warp = threadIdx.x / kWarp, lane = threadIdx.x & (kWarp - 1);
  if (threadIdx.x == 0) {
    for (int k = 0; k < 3; ++k) mbar_init(&bar[k], kWarp);
    abort_flag = 0;
  }
  __syncthreads();
  volatile int *af = &abort_flag;
  if (warp == 0) {
    mbar_arrive(&bar[2]);
    const bool acked = mbar_wait_warp(&bar[1], 0, af, limit);
    const bool ok = acked && mbar_wait_warp(&bar[0], 0, af, limit);
    if (lane == 0) out[0] = ok ? 1 : 0;
  } else {
    const bool seen = mbar_wait_warp(&bar[2], 0, af, limit);
    if (lane == 0) out[1] = seen ? 1 : 0;
    mbar_arrive(&bar[1]);
    const long long t0 = clock64();
    const bool ok = mbar_wait_warp(&bar[0], 0, af);
    const long long dt = clock64() - t0;
    if (lane == 0) { out[2] = ok ? 1 : 0; out[3] = dt; }
  }
  __syncthreads();
  if (threadIdx.x == 0) out[4] = abort_flag;
}

// ---- reference-semantics walk (FP64, one thread per target) ----

__device__ __forceinline__ void ref_pp(double bx, double by, double bz, double bm, double qp0,
                                       double qp1, double qp2, double mp, double G, double eps2,
                                       double &fx, double &fy, double &fz) {
  // morton_octree.f90:676-686
  const double dx = bx - qp0, dy = by - qp1, dz = bz - qp2;
  const double dist2 = dx * dx + dy * dy + dz * dz + eps2;
  double inv = 1.0 / sqrt(dist2);
  inv = inv * inv * inv;
  const double f = G * mp * bm * inv;
  fx = fx + f * dx; fy = fy + f * dy; fz = fz + f * dz;
}

template <int ORDER>
__global__ void __launch_bounds__(128)
reference_walk_kernel(WalkArgs a, const int64_t *__restrict__ targets, int64_t nt,
                      const int32_t *__restrict__ inv_perm, int64_t *__restrict__ counts) {
  const int L = a.sc->L;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nt;
       k += (int64_t)gridDim.x * blockDim.x) {
    if (targets && (targets[k] < 0 || targets[k] >= a.n)) {
      a.out[k] = a.out[nt + k] = a.out[2 * nt + k] = nan("");
      if (counts) counts[2 * k] = counts[2 * k + 1] = -1;
      continue;
    }
    const int p = targets ? inv_perm[targets[k]] : (int)k;
    const SysScalars &ss = a.ss[a.sys_of[p]];
    const double ssa = ss.ssa;
    const double4 q = a.spos[p];
    const double qp0 = q.x, qp1 = q.y, qp2 = q.z, mp = q.w;
    double fx = 0.0, fy = 0.0, fz = 0.0;
    int64_t npp = 0, npc = 0;
    // stack entries: node j >= 0; lone particle b as ~b (monopole at m q / m);
    // level-L lone particle b as ~b - 2^30 (summed at its exact position)
    int32_t st[8 * (kMaxDepth + 2) + 8];
    int top = 0;
    if (ss.root >= 0) st[top++] = ss.root;
    const int64_t max_pops = (int64_t)a.sc->n_compact + a.n + 8;
    int64_t pops = 0;
    while (top > 0) {
      if (++pops > max_pops) { atomicOr(&a.sc->err, kErrIndex); break; }
      const int32_t e = st[--top];
      if (e < 0) {
        const bool exact = e < -(1 << 30);
        const int b = exact ? ~(e + (1 << 30)) : ~e;
        if (b == p) continue;
        const double4 s = a.spos[b];
        if (exact) {
          ref_pp(s.x, s.y, s.z, s.w, qp0, qp1, qp2, mp, a.G, a.eps2, fx, fy, fz);
        } else {
          // single-particle node: qcm = (m q) / m (morton_octree.f90:446-458)
          const double cx = (s.w * s.x) / s.w, cy = (s.w * s.y) / s.w, cz = (s.w * s.z) / s.w;
          if (s.w > 0) ref_pp(cx, cy, cz, s.w, qp0, qp1, qp2, mp, a.G, a.eps2, fx, fy, fz);
        }
        ++npp;
        continue;
      }
      const int4 mt = a.meta[e];
      if (mt.w == 0) {  // level-L leaf: particle by particle (:672-691)
        for (int b = mt.x; b < mt.x + mt.y; ++b) {
          if (b == p) continue;
          const double4 s = a.spos[b];
          ref_pp(s.x, s.y, s.z, s.w, qp0, qp1, qp2, mp, a.G, a.eps2, fx, fy, fz);
          ++npp;
        }
        continue;
      }
      bool open = (mt.x <= p && p < mt.x + mt.y);  // :694-697
      if (!open) {
        const double4 c = a.com[e];
        const double dx = c.x - qp0, dy = c.y - qp1, dz = c.z - qp2;
        double dist2 = dx * dx + dy * dy + dz * dz;
        const double size = ssa * ldexp(1.0, -mt.z);
        if (size * size <= a.theta2 * dist2) {  // :706
          if (c.w > 0) {
            dist2 = dist2 + a.eps2;
            if (ORDER < 4) {
              double inv = 1.0 / sqrt(dist2);
              inv = inv * inv * inv;
              const double f = a.G * mp * c.w * inv;
              fx = fx + f * dx; fy = fy + f * dy; fz = fz + f * dz;
            } else {  // :721-753
              const double *Q = a.quad + 6 * (int64_t)e;
              const double invR = 1.0 / sqrt(dist2);
              const double invR2 = 1.0 / dist2;
              const double invR3 = invR * invR2;
              const double invR5 = invR3 * invR * invR;
              const double mx = dx * invR3 * c.w, my = dy * invR3 * c.w, mz = dz * invR3 * c.w;
              const double dx2 = 15.0 * dx * dx * invR2 - 3.0;
              const double dy2 = 15.0 * dy * dy * invR2 - 3.0;
              const double dz2 = 15.0 * dz * dz * invR2 - 3.0;
              const double dxyz = 15.0 * dx * dy * dz * invR2;
              double Qx = (Q[0] * (dx2 - 6.0) + Q[1] * dy2 + Q[2] * dz2) * 0.5 * dx;
              double Qy = (Q[1] * (dy2 - 6.0) + Q[2] * dz2 + Q[0] * dx2) * 0.5 * dy;
              double Qz = (Q[2] * (dz2 - 6.0) + Q[0] * dx2 + Q[1] * dy2) * 0.5 * dz;
              Qx = Qx + Q[3] * dy * dx2 + Q[4] * dz * dx2 + Q[5] * dxyz;
              Qy = Qy + Q[5] * dz * dy2 + Q[3] * dx * dy2 + Q[4] * dxyz;
              Qz = Qz + Q[4] * dx * dz2 + Q[5] * dy * dz2 + Q[3] * dxyz;
              if (ORDER < 8) {
                fx = fx + a.G * mp * (mx + invR5 * Qx);
                fy = fy + a.G * mp * (my + invR5 * Qy);
                fz = fz + a.G * mp * (mz + invR5 * Qz);
              } else {  // octupole terms of octree_default.f90:1012-1063
                const double *o = a.oct + 14 * (int64_t)e;
                const double invR7 = invR5 * invR * invR;
                const double invR9 = invR7 * invR * invR;
                double Ox = -1.5 * invR5 * o[11], Oy = -1.5 * invR5 * o[12], Oz = -1.5 * invR5 * o[13];
                double Oc = 7.5 * invR7 * (dx * o[11] + dy * o[12] + dz * o[13]);
                Ox = Ox + dx * Oc; Oy = Oy + dy * Oc; Oz = Oz + dz * Oc;
                const double ddx = dx * dx, ddy = dy * dy, ddz = dz * dz;
                Ox = Ox + 7.5 * invR7 * (ddx * o[0] + ddy * o[1] + ddz * o[2] + 2.0 * dx * dy * o[3] +
                                         2.0 * dx * dz * o[6] + 2.0 * dy * dz * o[9]);
                Oy = Oy + 7.5 * invR7 * (ddx * o[3] + ddy * o[4] + ddz * o[5] + 2.0 * dx * dy * o[1] +
                                         2.0 * dx * dz * o[9] + 2.0 * dy * dz * o[7]);
                Oz = Oz + 7.5 * invR7 * (ddx * o[6] + ddy * o[7] + ddz * o[8] + 2.0 * dx * dy * o[9] +
                                         2.0 * dx * dz * o[2] + 2.0 * dy * dz * o[5]);
                Oc = -17.5 * invR9 *
                     (ddx * dx * o[0] + ddy * dy * o[4] + ddz * dz * o[8] + 3.0 * ddx * dy * o[3] +
                      3.0 * ddx * dz * o[6] + 3.0 * ddy * dx * o[1] + 3.0 * ddy * dz * o[7] +
                      3.0 * ddz * dx * o[2] + 3.0 * ddz * dy * o[5] + 6.0 * dx * dy * dz * o[9]);
                Ox = Ox + dx * Oc; Oy = Oy + dy * Oc; Oz = Oz + dz * Oc;
                fx = fx + a.G * mp * (mx + invR5 * Qx + Ox);
                fy = fy + a.G * mp * (my + invR5 * Qy + Oy);
                fz = fz + a.G * mp * (mz + invR5 * Qz + Oz);
              }
            }
          }
          ++npc;
          continue;
        }
      }
      // open: push children in reverse so they pop in key order
      const bool deepest = (mt.z + 1 == L);
      for (int c = mt.w - 1; c >= 0; --c) {
        const int32_t ch = a.child[8 * (int64_t)e + c];
        if (top >= (int)(sizeof(st) / sizeof(st[0]))) break;
        st[top++] = (ch < 0 && deepest) ? ch - (1 << 30) : ch;
      }
    }
    double sc = 1.0;
    if (a.out_kind == 1) sc = 1.0 / mp;
    if (targets) {
      a.out[k] = fx * sc; a.out[nt + k] = fy * sc; a.out[2 * nt + k] = fz * sc;
    } else {
      double *out = a.out + 3 * ss.off;
      const int64_t orig = a.perm[p] - ss.off, ns = ss.n;
      out[orig] = fx * sc; out[ns + orig] = fy * sc; out[2 * ns + orig] = fz * sc;
    }
    if (counts) { counts[2 * k] = npp; counts[2 * k + 1] = npc; }
  }
}

int g_sm_count[64] = {0};

int sm_count() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (g_sm_count[dev] == 0) {
    int c = 0;
    cudaDeviceGetAttribute(&c, cudaDevAttrMultiProcessorCount, dev);
    g_sm_count[dev] = c > 0 ? c : 148;
  }
  return g_sm_count[dev];
}

}  // namespace

// stack slots: one per resident walk block of the FP32 walk (the most of any
// instantiation)
int64_t walk_slots() { return (int64_t)sm_count() * kWalkBlocksPerSm; }

int probe_bounded_wait(long long cycles, long long *out5) {
  long long *d = nullptr;
  if (cudaMalloc(&d, 5 * sizeof(long long)) != cudaSuccess) return 1;
  int rc = 0;
  if (cudaMemset(d, 0xff, 5 * sizeof(long long)) != cudaSuccess) rc = 1;
  if (!rc) {
    wait_probe_kernel<<<1, 2 * kWarp>>>(cycles, d);
    if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) rc = 1;
  }
  if (!rc && cudaMemcpy(out5, d, 5 * sizeof(long long), cudaMemcpyDeviceToHost) != cudaSuccess)
    rc = 1;
  cudaFree(d);
  return rc;
}

// The pipelined walk, when the kernel was built with the register count its
// setmaxnreg split assumes; returns false (nothing launched) otherwise.
template <int ORDER, int MAXTPL, bool SOFT>
static bool launch_pipe_walk(const WalkArgs &a, cudaStream_t s) {
  // the shared-memory limit is a per-device attribute: set it once per device
  static int per_sm[64] = {};
  const int smem = (int)sizeof(PipeSmem<ORDER>);
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) dev = 0;
  if (per_sm[dev] == 0) {
    cudaFuncAttributes fa{};
    cudaFuncGetAttributes(&fa, pipe_walk_kernel<ORDER, MAXTPL, SOFT>);
    cudaFuncSetAttribute(pipe_walk_kernel<ORDER, MAXTPL, SOFT>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    int v = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, pipe_walk_kernel<ORDER, MAXTPL, SOFT>,
                                                  kPipeThreads, smem);
    // a block launched with fewer registers than the split hands out would
    // wait for ever in setmaxnreg.inc: never launch it
    per_sm[dev] = (fa.numRegs == PipeRegs<ORDER>::regs && v > 0) ? v : -1;
  }
  if (per_sm[dev] < 0) return false;
  int64_t blocks = (int64_t)per_sm[dev] * sm_count();
  if (blocks * kTeams > a.slots) blocks = a.slots / kTeams;  // one stack per producer
  pipe_walk_kernel<ORDER, MAXTPL, SOFT><<<(unsigned)blocks, kPipeThreads, smem, s>>>(a);
  return true;
}

template <typename T, int ORDER, int MAXTPL, bool SOFT>
static void launch_group_walk(const WalkArgs &a, cudaStream_t s) {
  if (sizeof(T) == 4 && a.pipeline && launch_pipe_walk<ORDER, MAXTPL, SOFT>(a, s)) return;
  // exactly the blocks that are resident at once: no block waits for a
  // second wave behind the walk (which would also hold back other streams);
  // occupancy is a property of the device, so it is kept per device
  static int per_sm[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) dev = 0;
  if (per_sm[dev] == 0) {
    int v = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, group_walk_kernel<T, ORDER, MAXTPL, SOFT>,
                                                  kWarp, 0);
    per_sm[dev] = v > 0 ? v : 1;
  }
  int64_t blocks = (int64_t)per_sm[dev] * sm_count();
  if (blocks > a.slots) blocks = a.slots;
  group_walk_kernel<T, ORDER, MAXTPL, SOFT><<<(unsigned)blocks, kWarp, 0, s>>>(a);
}

static WalkArgs make_args(int64_t n, const WalkParams &p, Buffers &b, double *out) {
  WalkArgs a;
  a.meta = b.cn_meta; a.child = b.cn_child; a.com = b.cn_com; a.quad = b.cn_quad; a.oct = b.cn_oct;
  a.fq = b.cn_fq; a.fo = b.cn_fo; a.spos = b.spos; a.perm = b.v0; a.g_first = b.g_first;
  a.sys_of = b.sys_of; a.ss = b.ss;
  a.sc = b.sc; a.cursor = b.counters; a.stack = b.wstack; a.stack_cap = b.wstack_cap;
  a.slots = b.wstack_slots;
  a.stats = b.stats; a.out = out; a.n = n;
  a.theta2 = p.theta2; a.G = p.G; a.eps2 = p.eps2;
  a.out_kind = p.out_kind; a.leaf_cap = p.leaf_cap; a.count_stats = p.count_stats;
  a.mac = p.mac;
  a.g_begin = p.g_begin; a.g_end = p.g_end;
  a.pipeline = p.pipeline;
  return a;
}

template <typename T, int ORDER>
static void launch_walk_t(const WalkArgs &a, bool two, bool soft, cudaStream_t s) {
  if (two) {
    if (soft) launch_group_walk<T, ORDER, 2, true>(a, s);
    else launch_group_walk<T, ORDER, 2, false>(a, s);
  } else {
    if (soft) launch_group_walk<T, ORDER, 1, true>(a, s);
    else launch_group_walk<T, ORDER, 1, false>(a, s);
  }
}

void launch_walk(int64_t n, const WalkParams &p, Buffers &b, double *out, cudaStream_t s) {
  WalkArgs a = make_args(n, p, b, out);
  cudaMemsetAsync(b.counters, 0, sizeof(int32_t), s);
  const bool two = p.group_size > 32;
  const bool soft = p.eps2 > 0.0;
  if (p.precision == BH_PREC_FP64) {
    if (p.order >= 8) launch_walk_t<double, 8>(a, two, soft, s);
    else if (p.order >= 4) launch_walk_t<double, 4>(a, two, soft, s);
    else launch_walk_t<double, 1>(a, two, soft, s);
  } else {
    if (p.order >= 8) launch_walk_t<float, 8>(a, two, soft, s);
    else if (p.order >= 4) launch_walk_t<float, 4>(a, two, soft, s);
    else launch_walk_t<float, 1>(a, two, soft, s);
  }
}

__global__ void inv_perm_kernel(const int32_t *__restrict__ perm, int64_t n, int32_t *__restrict__ inv) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    inv[perm[i]] = (int32_t)i;
}

void launch_reference_walk(int64_t n, const WalkParams &p, Buffers &b, double *out,
                           const int64_t *targets, int64_t ntargets, int64_t *counts,
                           cudaStream_t s) {
  WalkArgs a = make_args(n, p, b, out);
  int32_t *inv = nullptr;
  if (targets) {
    inv = b.gscan;  // free after the group pass
    inv_perm_kernel<<<grid_for(n, 256, 148 * 8), 256, 0, s>>>(b.v0, n, inv);
  }
  const int64_t nt = targets ? ntargets : n;
  const int grid = grid_for(nt, 128, 148 * 32);
  if (p.order >= 8)
    reference_walk_kernel<8><<<grid, 128, 0, s>>>(a, targets, nt, inv, counts);
  else if (p.order >= 4)
    reference_walk_kernel<4><<<grid, 128, 0, s>>>(a, targets, nt, inv, counts);
  else
    reference_walk_kernel<1><<<grid, 128, 0, s>>>(a, targets, nt, inv, counts);
}

}  // namespace bh
