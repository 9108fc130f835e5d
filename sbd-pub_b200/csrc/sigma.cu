// sigma = H*C on the GPU (separated sign convention; see tpb_common.cuh).
//
// Replaces MultTPBThrust::run (tpb/mult_thrust.h:1172-1582) and sbd::mult (tpb/mult.h:625-881).
// Where the reference launches one thread per (connection, determinant) and adds into sigma with
// FP64 atomics, every sigma element here has exactly one owner, so results are deterministic:
//
//   alpha pass    sigma[Ia, Ib] = (H_ii - shift) C[Ia, Ib] + sum_Ja H_a(Ia, Ja) C[Ja, Ib]
//                 (+ the alpha-single x beta-single terms sa sb (pq|rs) C[Ja, Jb] when the
//                 singles are sparse), gathering rows Ja of C from an L2-resident column slab;
//                 the same CTA writes its own tile of C transposed into C^T.
//   beta pass     sigma[Ia, Ib] += sum_Jb H_b(Ib, Jb) C^T[Jb, Ia], the same kernel on C^T, its
//                 result transposed back through shared memory with coalesced writes.
// Both passes are the alpha-string "row SpMM" on a row-major operand, which is what makes every
// gather a 128-byte coalesced row segment.
//
// The alpha-beta term of FCI-like problems (dense singles) goes through the gather -> dense
// (pq|rs) contraction -> scatter path in ab_dense.cu instead of the direct loop.
#include <algorithm>
#include <string>

#include "tpb_common.cuh"
#include "vecops.cuh"

namespace sbdtpb {
namespace {

constexpr int kBlkRows = 8;  // bra rows per CTA
constexpr int kBlkThreads = 128;
// Thread mapping of a CTA per element type and pass: the 128 threads form G row groups, each
// thread holding kBlkRows / G rows of VW columns (fewer accumulators per thread for larger G, so
// more CTAs fit an SM), with the register budget of M CTAs per SM; OS parks the C values the alpha
// pass writes out transposed in shared memory instead of registers.  Measured with the singles'
// Coulomb sums read from the per-pair table as 16-byte loads, ms per pass at 4e8 determinants
// (norb=32) / 1e8 (norb=28) / norb=12 FCI: FP32 alpha 2/8/OS 3.31 / 1.45 (2/7: 3.59 / 1.48,
// 2/8: 3.66 / 1.52, 1/6/OS: 3.77 / 1.50, 2/9/OS spills: 3.84 / 1.78); FP32 beta 2/8 3.35 / 1.36 /
// 0.159 (2/9: 3.38 / 1.44 / 0.185, 2/10: 3.68 / 1.63, 4/10: 14.4); FP64 alpha 2/7 6.39 / 2.53 /
// 0.187 (2/8: 6.44, 2/7/OS: 6.45, 2/6: 6.95); FP64 beta 2/9 5.76 / 2.71 / 0.196 (2/8: 5.93 / 2.38 /
// 0.197, 2/10: 6.09).  Four groups lose the 16-byte runs of the FP32 transposed write-out.  Small
// problems run the FP32 alpha pass with 2/6 and no parking (norb=12 FCI 0.154 ms; 2/7: 0.159,
// 2/7/OS: 0.161, 2/8/OS: 0.170, 1/5: 0.279); the switch is at 10,000 one-group CTAs.
// The mapping of a pass as template arguments: G row groups, register budget of M CTAs per SM.
template <typename T>
__device__ __forceinline__ T val_of(const double *v, const float *vf, uint32_t e);
template <>
__device__ __forceinline__ double val_of<double>(const double *v, const float *, uint32_t e) {
  return __ldg(&v[e]);
}
template <>
__device__ __forceinline__ float val_of<float>(const double *, const float *vf, uint32_t e) {
  return __ldg(&vf[e]);
}

// The element arithmetic of every sigma pass, written out so that each kernel form rounds the same
// way (no contraction left to the compiler): doubles term acc + v x as one fused multiply-add, the
// singles term and the diagonal as a rounded FP64 product added to the accumulator.
__device__ __forceinline__ float madd(float acc, float v, float x) { return __fmaf_rn(v, x, acc); }
__device__ __forceinline__ double madd(double acc, double v, double x) { return __fma_rn(v, x, acc); }

// VW consecutive elements of type T: one 16-byte load when kVec, VW scalars otherwise.
template <typename T, int VW, bool kVec>
struct Vec;
template <bool kVec>
struct Vec<float, 4, kVec> {
  float v[4];
  __device__ __forceinline__ void store(float *p) const {
    *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
  }
  // coherent load of data this kernel also writes
  __device__ __forceinline__ void load_rw(const float *p) {
    const float4 f = *reinterpret_cast<const float4 *>(p);
    v[0] = f.x, v[1] = f.y, v[2] = f.z, v[3] = f.w;
  }
  __device__ __forceinline__ void load(const float *p) {
    if (kVec) {
      const float4 f = __ldg(reinterpret_cast<const float4 *>(p));
      v[0] = f.x, v[1] = f.y, v[2] = f.z, v[3] = f.w;
    } else {
#pragma unroll
      for (int i = 0; i < 4; i++) v[i] = __ldg(p + i);
    }
  }
};
template <bool kVec>
struct Vec<double, 2, kVec> {
  double v[2];
  __device__ __forceinline__ void store(double *p) const {
    *reinterpret_cast<double2 *>(p) = make_double2(v[0], v[1]);
  }
  __device__ __forceinline__ void load_rw(const double *p) {
    const double2 f = *reinterpret_cast<const double2 *>(p);
    v[0] = f.x, v[1] = f.y;
  }
  __device__ __forceinline__ void load(const double *p) {
    if (kVec) {
      const double2 f = __ldg(reinterpret_cast<const double2 *>(p));
      v[0] = f.x, v[1] = f.y;
    } else {
      v[0] = __ldg(p);
      v[1] = __ldg(p + 1);
    }
  }
};

struct BlockArgs {
  // sigma program of the bra spin (rows of X)
  const uint32_t *s_off, *s_ket;
  const double *s_val;
  const float *s_valf;
  const int32_t *s_pair;
  const uint32_t *d_off, *d_ket;
  const double *d_val;
  const float *d_valf;
  const uint64_t *col_str;  // strings of the column spin (other-spin Coulomb term of singles)
  const double *jtab;       // per-pair Coulomb sums over those strings (SigmaProg::jtab), or null
                            // (then the singles loop over the column string's orbitals)
  const int32_t *pmap;      // pair -> row of jtab
  const double *vd;         // (pq|kk) [L*L][L]
  int L;
  uint32_t nrows, ncols;    // X is nrows x ncols, row-major
  uint32_t max_d, max_s;    // most doubles / singles entries of any kBlkRows-row block
  // alpha pass only: diagonal (H_ii = I0 + E(Ia) + E(Ib) + sum_{q in Ib} uJ[Ia][q]) and the
  // alpha-single x beta-single terms
  double core_shift;     // FP64 pass: shift; FP32 pass: H_00 - shift
  const double *hii;     // FP64 diagonal
  const float *hii32;    // H_ii - H_00 in FP32
  const double *Ea, *Eb, *uJ;
  int accumulate;
  int do_ab;
  const uint32_t *bs_off, *bs_ket;
  const int32_t *bs_pair;
  const double *eri;
};

// One kernel, two passes.  A CTA owns kBlkRows consecutive bra strings (rows of X) and a slab of
// (kBlkThreads / G) * VW columns; its threads form G row groups, each thread VW consecutive
// columns (one 16-byte access when the row length allows it) of kBlkRows / G rows.  Blocks run
// slab-major so the CTAs in flight gather from one slab of X that stays in L2.  The block's table
// entries (one contiguous CSR range) are staged in shared memory first, so the gathers
// X[ket, cols] issue back to back.
//   alpha pass (kAlpha): X = C.  Adds the diagonal (and, in the allocation-free path only, the
//     alpha-single x beta-single terms, which otherwise have kernels of their own) and writes
//     sigma[Ia, Ib] once; the thread's own C[Ia-block, cols] values go out transposed to C^T as
//     contiguous runs of its rows.  Singles read the other spin's Coulomb sums from the per-pair
//     table when it exists (16-byte loads for a whole column group), else loop over the column
//     string's orbitals.
//   beta pass: X = C^T.  Each thread adds its rows x VW results into sigma[Ia, Ib0 ...)
//     (contiguous along Ib) for its columns Ia.
//   symmetric alpha pass (kSym, with kAlpha): for C = C^T over identical alpha and beta strings the
//     beta part of sigma is the transpose of the alpha part, so the pass writes
//     B = (H_ii - shift) C / 2 + (alpha part) and no C^T; sym_add then forms sigma = B + B^T.
template <typename T, bool kAlpha, bool kVec, int G, int M, bool OS, bool kSym = false>
__global__ void __launch_bounds__(kBlkThreads, M)
    sigma_block_kernel(BlockArgs a, const T *__restrict__ X, T *__restrict__ out, T *__restrict__ XT) {
  constexpr int VW = 16 / sizeof(T);
  constexpr int TC = kBlkThreads / G;  // threads across the columns of the slab
  constexpr int RPT = kBlkRows / G;    // rows per thread
  constexpr int W = TC * VW;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint32_t *sd_ket = reinterpret_cast<uint32_t *>(smem_raw);
  T *sd_val = reinterpret_cast<T *>(smem_raw + ((a.max_d * 4 + 15) & ~15u));
  unsigned char *sp = smem_raw + ((a.max_d * 4 + 15) & ~15u) + a.max_d * sizeof(T);
  sp = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(sp) + 15) & ~(uintptr_t)15);
  uint32_t *ss_ket = reinterpret_cast<uint32_t *>(sp);
  int32_t *ss_pair = reinterpret_cast<int32_t *>(sp + a.max_s * 4);
  double *ss_val = reinterpret_cast<double *>(sp + ((a.max_s * 8 + 15) & ~15u));
  // OS: the alpha pass parks its own C values for the transposed write-out in shared memory
  // ([row][column of the thread][thread], conflict-free) instead of registers
  T *own_s = reinterpret_cast<T *>(
      (reinterpret_cast<uintptr_t>(ss_val + a.max_s) + 15) & ~(uintptr_t)15);

  const uint32_t nrb = (a.nrows + kBlkRows - 1) / kBlkRows;
  const uint32_t rb = blockIdx.x % nrb, slab = blockIdx.x / nrb;
  const uint32_t r0 = rb * kBlkRows;
  const uint32_t ncols = a.ncols;
  const int L = a.L, L2 = L * L;
  const int nr = (int)min((uint32_t)kBlkRows, a.nrows - r0);
  const int grp = threadIdx.x / TC;                                  // row group of this thread
  const uint32_t cbase = slab * W + (threadIdx.x % TC) * VW;         // first of its VW columns

  // stage the block's table entries
  const uint32_t dlo = __ldg(&a.d_off[r0]), dhi = __ldg(&a.d_off[r0 + nr]);
  const uint32_t slo = __ldg(&a.s_off[r0]), shi = __ldg(&a.s_off[r0 + nr]);
  for (uint32_t e = dlo + threadIdx.x; e < dhi; e += blockDim.x) {
    sd_ket[e - dlo] = __ldg(&a.d_ket[e]);
    sd_val[e - dlo] = val_of<T>(a.d_val, a.d_valf, e);
  }
  for (uint32_t e = slo + threadIdx.x; e < shi; e += blockDim.x) {
    ss_ket[e - slo] = __ldg(&a.s_ket[e]);
    ss_pair[e - slo] = __ldg(&a.s_pair[e]);
    ss_val[e - slo] = (double)val_of<T>(a.s_val, a.s_valf, e);
  }
  __syncthreads();

  bool ok[VW];
  uint64_t cstr[VW];
#pragma unroll
  for (int i = 0; i < VW; i++) {
    ok[i] = cbase + i < ncols;
    cstr[i] = ok[i] ? __ldg(&a.col_str[cbase + i]) : 0ull;
  }
  const bool any = ok[0];
  const bool full = ok[VW - 1];

  T acc[RPT][VW];
  T own[(kAlpha && !OS && !kSym) ? RPT : 1][VW];
#pragma unroll
  for (int r = 0; r < RPT; r++) {
#pragma unroll
    for (int i = 0; i < VW; i++) {
      acc[r][i] = T(0);
      if (kAlpha && !OS && !kSym) own[r][i] = T(0);
    }
  }
  const int rlo = grp * RPT;  // this thread's rows: r0 + rlo .. r0 + rlo + RPT
#pragma unroll
  for (int r = 0; r < RPT; r++) {
    if (rlo + r >= nr || !any) continue;
    const uint32_t row = r0 + rlo + r;
    const uint32_t d0 = __ldg(&a.d_off[row]) - dlo, d1 = __ldg(&a.d_off[row + 1]) - dlo;
#pragma unroll 4
    for (uint32_t e = d0; e < d1; e++) {
      const T v = sd_val[e];
      const T *xr = X + (size_t)sd_ket[e] * ncols + cbase;
      Vec<T, VW, kVec> x;
      if (kVec && full) {
        x.load(xr);
      } else {
#pragma unroll
        for (int i = 0; i < VW; i++) x.v[i] = ok[i] ? __ldg(xr + i) : T(0);
      }
#pragma unroll
      for (int i = 0; i < VW; i++) acc[r][i] = madd(acc[r][i], v, x.v[i]);
    }
    const uint32_t s0 = __ldg(&a.s_off[row]) - slo, s1 = __ldg(&a.s_off[row + 1]) - slo;
    for (uint32_t e = s0; e < s1; e++) {
      const uint32_t ket = ss_ket[e];
      const double v = ss_val[e];
      const int32_t ps = ss_pair[e];
      const int pr = (ps > 0 ? ps : -ps) - 1;
      const double sg = ps > 0 ? 1.0 : -1.0;
      const double *vrow = a.vd + (size_t)pr * L;
      const T *xr = X + (size_t)ket * ncols;
      const double *jr = a.jtab ? a.jtab + (size_t)__ldg(&a.pmap[pr]) * ncols : nullptr;
      if (kVec && full && jr && !a.do_ab) {
        // whole 16-byte column group: the ket values and the table's Coulomb sums as vector
        // loads (table rows are ncols doubles, ncols a multiple of VW, so jr + cbase is aligned)
        Vec<T, VW, true> xv;
        xv.load(xr + cbase);
        double o[VW];
#pragma unroll
        for (int i = 0; i < VW; i += 2) {
          const double2 jj = __ldg(reinterpret_cast<const double2 *>(jr + cbase + i));
          o[i] = jj.x;
          o[i + 1] = jj.y;
        }
#pragma unroll
        for (int i = 0; i < VW; i++) acc[r][i] += (T)__dmul_rn(v + sg * o[i], (double)xv.v[i]);
        continue;
      }
#pragma unroll
      for (int i = 0; i < VW; i++) {
        if (!ok[i]) continue;
        const uint32_t c = cbase + i;
        double o = 0.0;
        if (jr) {
          o = __ldg(&jr[c]);
        } else {
          uint64_t occ = cstr[i];
          while (occ) {
            o += __ldg(&vrow[lowest_bit(occ)]);
            occ &= occ - 1;
          }
        }
        double x = __dmul_rn(v + sg * o, (double)__ldg(&xr[c]));
        if (kAlpha && a.do_ab) {
          // this alpha single (ket = Ja, pair pr, sign sg) x every beta single of column Ib
          const uint32_t f1 = __ldg(&a.bs_off[c + 1]);
          for (uint32_t f = __ldg(&a.bs_off[c]); f < f1; f++) {
            const int32_t pb = __ldg(&a.bs_pair[f]);
            const int rs = (pb > 0 ? pb : -pb) - 1;
            const double g = __ldg(&a.eri[(size_t)pr * L2 + rs]);
            const double cj = (double)__ldg(&xr[__ldg(&a.bs_ket[f])]);
            x += (pb > 0 ? g : -g) * cj * sg;
          }
        }
        acc[r][i] += (T)x;
      }
    }
    if (kAlpha) {
      // H_ii - shift: FP64 diagonal for the FP64 pass, (H_ii - H_00) in FP32 plus the FP64
      // constant H_00 - shift for the FP32 pass
      const size_t idx = (size_t)row * ncols + cbase;
      const T *hsrc = sizeof(T) == 8 ? reinterpret_cast<const T *>(a.hii) : reinterpret_cast<const T *>(a.hii32);
      const double hshift = sizeof(T) == 8 ? -a.core_shift : a.core_shift;
      Vec<T, VW, kVec> xo, hv, ov;
      if (kVec && full) {
        xo.load(X + idx);
        hv.load(hsrc + idx);
        if (a.accumulate) ov.load_rw(out + idx);
      } else {
#pragma unroll
        for (int i = 0; i < VW; i++) {
          xo.v[i] = ok[i] ? __ldg(X + idx + i) : T(0);
          hv.v[i] = ok[i] ? __ldg(hsrc + idx + i) : T(0);
          ov.v[i] = (ok[i] && a.accumulate) ? out[idx + i] : T(0);
        }
      }
#pragma unroll
      for (int i = 0; i < VW; i++) {
        double res;
        if constexpr (kSym) {
          res = (double)acc[r][i] + 0.5 * __dmul_rn((double)hv.v[i] + hshift, (double)xo.v[i]);
        } else {
          if (OS) own_s[(r * VW + i) * kBlkThreads + threadIdx.x] = xo.v[i];
          else own[r][i] = xo.v[i];
          res = (double)acc[r][i] + __dmul_rn((double)hv.v[i] + hshift, (double)xo.v[i]);
        }
        if (a.accumulate) res += (double)ov.v[i];
        ov.v[i] = (T)res;
      }
      if (kVec && full) {
        ov.store(out + idx);
      } else {
#pragma unroll
        for (int i = 0; i < VW; i++)
          if (ok[i]) out[idx + i] = ov.v[i];
      }
    }
  }
  if constexpr (kSym) return;  // B only: no C^T
  // transposed write-out: column c gets this thread's rows contiguous (index c * nrows + r), as
  // 16-byte accesses when the block is full and every column starts 16-byte aligned
  constexpr int RW = 16 / sizeof(T);
  constexpr bool kRuns = RPT % RW == 0;  // the thread's rows form whole 16-byte runs
  const bool vec_out = kRuns && kVec && nr == kBlkRows && (a.nrows % RW) == 0;
#pragma unroll
  for (int i = 0; i < VW; i++) {
    if (!ok[i]) continue;
    const size_t o = (size_t)(cbase + i) * a.nrows + r0 + rlo;
    if constexpr (kRuns) {
      if (vec_out) {
#pragma unroll
        for (int r = 0; r < RPT; r += RW) {
          Vec<T, RW, true> v;
          if (kAlpha) {
#pragma unroll
            for (int q = 0; q < RW; q++)
              v.v[q] = OS ? own_s[((r + q) * VW + i) * kBlkThreads + threadIdx.x] : own[OS ? 0 : r + q][i];
          } else {
            v.load_rw(out + o + r);
#pragma unroll
            for (int q = 0; q < RW; q++) v.v[q] += acc[r + q][i];
          }
          v.store(kAlpha ? XT + o + r : out + o + r);
        }
        continue;
      }
    }
    {
#pragma unroll
      for (int r = 0; r < RPT; r++) {
        if (rlo + r < nr) {
          if (kAlpha) XT[o + r] = OS ? own_s[(r * VW + i) * kBlkThreads + threadIdx.x] : own[OS ? 0 : r][i];
          else out[o + r] += acc[r][i];
        }
      }
    }
  }
}

// Alpha-single x beta-single terms when both singles tables are sparse:
//   sigma[Ia, Ib] += sum_{(Ja, pq, sa) in S_a(Ia)} sum_{(Jb, rs, sb) in S_b(Ib)} sa sb (pq|rs) C[Ja, Jb]
// One CTA per alpha row Ia that has singles.  For a group of its singles the CTA stages in shared
// memory the ket rows C[Ja] -- only the columns Jb that are kets of some beta single, compacted
// (kets[] lists them ascending; the beta program addresses them by position), and of those one
// range at a time -- and the integral rows sa (pq|.) (sign folded in), so the scattered reads
// C[Ja, Jb] and (pq|rs) at the beta singles are shared-memory reads; each thread owns a set of beta
// columns Ib that have singles and adds its sum over the range's entries into sigma[Ia, Ib] once
// per group.  Every group re-reads the beta program's part for its range, so the ranges are made
// short enough (on dense singles) for groups of several singles at two CTAs per SM; with sparse
// singles there is one range and four CTAs per SM.  Sums in the vector type (FP32 vectors: FP32
// products and sums, like the other FP32 sigma terms).  Without room for one staged row (kStage
// false) the same loop reads C and the integrals through L1/L2.
struct AbSparseArgs {
  const uint32_t *rows;  // alpha rows with at least one single
  const uint2 *colp;     // per ket range: (column, first entry) of each beta column with singles, then (0, range end)
  const uint2 *bsp;      // beta singles entries: (position of the ket in kets, +-(rs + 1) with the beta sign)
  const uint32_t *kets;  // [nk] the distinct kets of the beta singles, ascending
  uint32_t nk;
  uint32_t ncols_s;
  uint32_t nchunks, chunk;  // ket ranges (program parts) and kets per range
  const uint32_t *as_off, *as_ket;
  const int32_t *as_pair;  // +-(pq + 1), sign = alpha sign
  const double *eri;       // (pq|rs) [L*L][L*L]
  int L2;
  uint32_t nb;     // row length of C and sigma
  uint32_t group;  // singles staged per round
  double scale;    // weight of the term
  int upper;       // only columns Ib >= Ia (weight 1/2 on Ib == Ia): the symmetric sigma's B
};

template <typename T, bool kStage, bool kRanges>
__global__ void __launch_bounds__(256)
    ab_sparse_kernel(AbSparseArgs a, const T *__restrict__ C, T *__restrict__ sigma) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *rows = reinterpret_cast<T *>(smem_raw);                // [group][chunk]
  T *gint = rows + (size_t)a.group * a.chunk;               // [group][L2], sign folded in
  const uint32_t ia = __ldg(&a.rows[blockIdx.x]);
  const uint32_t e0 = __ldg(&a.as_off[ia]), e1 = __ldg(&a.as_off[ia + 1]);
  T *srow = sigma + (size_t)ia * a.nb;
  const uint32_t nchunks = kRanges ? a.nchunks : 1;
  for (uint32_t m = 0; m < nchunks; m++) {
    const uint32_t k0 = kRanges ? m * a.chunk : 0, nkm = kRanges ? min(a.nk, k0 + a.chunk) - k0 : a.nk;
    const uint2 *colp = kRanges ? a.colp + (size_t)m * (a.ncols_s + 1) : a.colp;
    for (uint32_t g0 = e0; g0 < e1; g0 += a.group) {
      const uint32_t g1 = min(e1, g0 + a.group), ng = g1 - g0;
      if (kStage) {
        __syncthreads();
        for (uint32_t j = 0; j < ng; j++) {
          const T *src = C + (size_t)__ldg(&a.as_ket[g0 + j]) * a.nb;
          T *dst = rows + (size_t)j * a.chunk;
          for (uint32_t c = threadIdx.x; c < nkm; c += blockDim.x) dst[c] = __ldg(&src[__ldg(&a.kets[k0 + c])]);
          const int32_t pa = __ldg(&a.as_pair[g0 + j]);
          const double *erow = a.eri + (size_t)((pa > 0 ? pa : -pa) - 1) * a.L2;
          T *gdst = gint + (size_t)j * a.L2;
          for (int c = threadIdx.x; c < a.L2; c += blockDim.x) {
            const double g = __ldg(&erow[c]);
            gdst[c] = (T)(pa > 0 ? g : -g);
          }
        }
        __syncthreads();
      }
      // sum over the beta singles of compact column q in this ket range (its column index in ib;
      // false when the range has none of them)
      auto column = [&](uint32_t q, uint32_t &ib, double &out) -> bool {
        const uint2 c0 = __ldg(&colp[q]), c1 = __ldg(&colp[q + 1]);
        ib = c0.x;
        T acc = 0;
        for (uint32_t f = c0.y; f < c1.y; f++) {
          const uint2 be = __ldg(&a.bsp[f]);
          const uint32_t jb = be.x - k0;
          const int32_t pb = (int32_t)be.y;
          const int rs = (pb > 0 ? pb : -pb) - 1;
          T sum = 0;
          for (uint32_t j = 0; j < ng; j++) {
            if (kStage) {
              sum = madd(sum, gint[(size_t)j * a.L2 + rs], rows[(size_t)j * a.chunk + jb]);
            } else {
              const int32_t pa = __ldg(&a.as_pair[g0 + j]);
              const T g = (T)__ldg(&a.eri[(size_t)((pa > 0 ? pa : -pa) - 1) * a.L2 + rs]);
              sum = madd(sum, pa > 0 ? g : -g, __ldg(&C[(size_t)__ldg(&a.as_ket[g0 + j]) * a.nb + __ldg(&a.kets[be.x])]));
            }
          }
          acc += pb > 0 ? sum : -sum;
        }
        out = (double)acc;
        return !kRanges || c1.y > c0.y;
      };
      // two independent columns per iteration, so their load chains overlap
      uint32_t q = threadIdx.x;
      for (; q + blockDim.x < a.ncols_s; q += 2 * blockDim.x) {
        uint32_t ib0, ib1;
        double s0, s1;
        if (a.upper) {
          // the symmetric sigma's B: columns Ib >= Ia only (B + B^T restores the rest), the diagonal
          // at half weight
          const uint32_t c0 = __ldg(&colp[q]).x, c1 = __ldg(&colp[q + blockDim.x]).x;
          const bool u0 = c0 >= ia, u1 = c1 >= ia;
          if (!u0 && !u1) continue;
          if (u0 && u1) {
            const bool h0 = column(q, ib0, s0), h1 = column(q + blockDim.x, ib1, s1);
            const T o0 = h0 ? srow[ib0] : T(0), o1 = h1 ? srow[ib1] : T(0);
            if (h0) srow[ib0] = (T)((double)o0 + (ib0 == ia ? 0.5 : 1.0) * a.scale * s0);
            if (h1) srow[ib1] = (T)((double)o1 + (ib1 == ia ? 0.5 : 1.0) * a.scale * s1);
          } else {
            const uint32_t qq = u0 ? q : q + blockDim.x;
            if (column(qq, ib0, s0)) srow[ib0] = (T)((double)srow[ib0] + (ib0 == ia ? 0.5 : 1.0) * a.scale * s0);
          }
          continue;
        }
        const bool h0 = column(q, ib0, s0), h1 = column(q + blockDim.x, ib1, s1);
        const T o0 = h0 ? srow[ib0] : T(0), o1 = h1 ? srow[ib1] : T(0);  // both loads before the stores
        if (h0) srow[ib0] = (T)((double)o0 + a.scale * s0);
        if (h1) srow[ib1] = (T)((double)o1 + a.scale * s1);
      }
      if (q < a.ncols_s && (!a.upper || __ldg(&colp[q]).x >= ia)) {
        uint32_t ib0;
        double s0;
        if (column(q, ib0, s0))
          srow[ib0] = (T)((double)srow[ib0] + (a.upper && ib0 == ia ? 0.5 : 1.0) * a.scale * s0);
      }
    }
  }
}

__global__ void reorder_sign_kernel_f64(const uint64_t *__restrict__ apar,
                                        const uint64_t *__restrict__ bstr, uint32_t nb, size_t n,
                                        const double *__restrict__ x, double *__restrict__ y) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const size_t ia = i / nb, ib = i - ia * nb;
    const double v = x[i];
    y[i] = (__popcll(apar[ia] & bstr[ib]) & 1) ? -v : v;
  }
}

__global__ void reorder_sign_kernel_f32(const uint64_t *__restrict__ apar,
                                        const uint64_t *__restrict__ bstr, uint32_t nb, size_t n,
                                        const float *__restrict__ x, float *__restrict__ y) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const size_t ia = i / nb, ib = i - ia * nb;
    const float v = x[i];
    y[i] = (__popcll(apar[ia] & bstr[ib]) & 1) ? -v : v;
  }
}

// The general alpha and beta passes with CM column groups per thread, as sigma_sym_cm_kernel does
// for the one-pass form: each thread covers CM 16-byte column groups TC * VW columns apart and reuses
// each staged table entry for all of them.  16-byte rows and no alpha-single x beta-single terms
// (the caller falls back to sigma_block_kernel otherwise).  The alpha pass (X = C) adds the diagonal,
// writes sigma once and its own C values transposed into C^T (parked in shared memory when OS); the
// beta pass (X = C^T) adds its sums into sigma transposed.  Same per-element arithmetic and order
// as sigma_block_kernel, so the same bits.
template <typename T, bool kAlpha, int G, int M, int CM, bool OS>
__global__ void __launch_bounds__(kBlkThreads, M)
    sigma_pass_cm_kernel(BlockArgs a, const T *__restrict__ X, T *__restrict__ out, T *__restrict__ XT) {
  constexpr int VW = 16 / sizeof(T);
  constexpr int TC = kBlkThreads / G;
  constexpr int RPT = kBlkRows / G;
  constexpr int W = CM * TC * VW;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint32_t *sd_ket = reinterpret_cast<uint32_t *>(smem_raw);
  T *sd_val = reinterpret_cast<T *>(smem_raw + ((a.max_d * 4 + 15) & ~15u));
  unsigned char *sp = smem_raw + ((a.max_d * 4 + 15) & ~15u) + a.max_d * sizeof(T);
  sp = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(sp) + 15) & ~(uintptr_t)15);
  uint32_t *ss_ket = reinterpret_cast<uint32_t *>(sp);
  int32_t *ss_pair = reinterpret_cast<int32_t *>(sp + a.max_s * 4);
  double *ss_val = reinterpret_cast<double *>(sp + ((a.max_s * 8 + 15) & ~15u));
  // OS: [row][column group][element][thread], conflict-free
  T *own_s = reinterpret_cast<T *>((reinterpret_cast<uintptr_t>(ss_val + a.max_s) + 15) & ~(uintptr_t)15);

  const uint32_t nrb = (a.nrows + kBlkRows - 1) / kBlkRows;
  const uint32_t rb = blockIdx.x % nrb, slab = blockIdx.x / nrb;
  const uint32_t r0 = rb * kBlkRows;
  const uint32_t ncols = a.ncols;
  const int nr = (int)min((uint32_t)kBlkRows, a.nrows - r0);
  const int grp = threadIdx.x / TC;
  uint32_t cb[CM];
  bool full[CM];
#pragma unroll
  for (int g = 0; g < CM; g++) {
    cb[g] = slab * W + g * TC * VW + (threadIdx.x % TC) * VW;
    full[g] = cb[g] + VW <= ncols;  // ncols is a multiple of VW: a group is all in or all out
  }

  const uint32_t dlo = __ldg(&a.d_off[r0]), dhi = __ldg(&a.d_off[r0 + nr]);
  const uint32_t slo = __ldg(&a.s_off[r0]), shi = __ldg(&a.s_off[r0 + nr]);
  for (uint32_t e = dlo + threadIdx.x; e < dhi; e += blockDim.x) {
    sd_ket[e - dlo] = __ldg(&a.d_ket[e]);
    sd_val[e - dlo] = val_of<T>(a.d_val, a.d_valf, e);
  }
  for (uint32_t e = slo + threadIdx.x; e < shi; e += blockDim.x) {
    ss_ket[e - slo] = __ldg(&a.s_ket[e]);
    ss_pair[e - slo] = __ldg(&a.s_pair[e]);
    ss_val[e - slo] = (double)val_of<T>(a.s_val, a.s_valf, e);
  }
  __syncthreads();
  if (!full[0]) return;

  T acc[RPT][CM][VW];
  T own[(kAlpha && !OS) ? RPT : 1][CM][VW];
#pragma unroll
  for (int r = 0; r < RPT; r++)
#pragma unroll
    for (int g = 0; g < CM; g++)
#pragma unroll
      for (int i = 0; i < VW; i++) {
        acc[r][g][i] = T(0);
        if (kAlpha && !OS) own[r][g][i] = T(0);
      }
  const int rlo = grp * RPT;
#pragma unroll
  for (int r = 0; r < RPT; r++) {
    if (rlo + r >= nr) continue;
    const uint32_t row = r0 + rlo + r;
    const uint32_t d0 = __ldg(&a.d_off[row]) - dlo, d1 = __ldg(&a.d_off[row + 1]) - dlo;
#pragma unroll 4
    for (uint32_t e = d0; e < d1; e++) {
      const T v = sd_val[e];
      const T *xr = X + (size_t)sd_ket[e] * ncols;
#pragma unroll
      for (int g = 0; g < CM; g++) {
        if (g > 0 && !full[g]) continue;
        Vec<T, VW, true> x;
        x.load(xr + cb[g]);
#pragma unroll
        for (int i = 0; i < VW; i++) acc[r][g][i] = madd(acc[r][g][i], v, x.v[i]);
      }
    }
    const uint32_t s0 = __ldg(&a.s_off[row]) - slo, s1 = __ldg(&a.s_off[row + 1]) - slo;
    for (uint32_t e = s0; e < s1; e++) {
      const uint32_t ket = ss_ket[e];
      const double v = ss_val[e];
      const int32_t ps = ss_pair[e];
      const int pr = (ps > 0 ? ps : -ps) - 1;
      const double sg = ps > 0 ? 1.0 : -1.0;
      const double *vrow = a.vd + (size_t)pr * a.L;
      const T *xr = X + (size_t)ket * ncols;
      const double *jr = a.jtab ? a.jtab + (size_t)__ldg(&a.pmap[pr]) * ncols : nullptr;
#pragma unroll
      for (int g = 0; g < CM; g++) {
        if (g > 0 && !full[g]) continue;
        Vec<T, VW, true> xv;
        xv.load(xr + cb[g]);
        double o[VW];
        if (jr) {
#pragma unroll
          for (int i = 0; i < VW; i += 2) {
            const double2 jj = __ldg(reinterpret_cast<const double2 *>(jr + cb[g] + i));
            o[i] = jj.x;
            o[i + 1] = jj.y;
          }
        } else {
#pragma unroll
          for (int i = 0; i < VW; i++) {
            uint64_t occ = __ldg(&a.col_str[cb[g] + i]);
            o[i] = 0.0;
            while (occ) {
              o[i] += __ldg(&vrow[lowest_bit(occ)]);
              occ &= occ - 1;
            }
          }
        }
#pragma unroll
        for (int i = 0; i < VW; i++) acc[r][g][i] += (T)__dmul_rn(v + sg * o[i], (double)xv.v[i]);
      }
    }
    if constexpr (kAlpha) {
      const T *hsrc = sizeof(T) == 8 ? reinterpret_cast<const T *>(a.hii) : reinterpret_cast<const T *>(a.hii32);
      const double hshift = sizeof(T) == 8 ? -a.core_shift : a.core_shift;
#pragma unroll
      for (int g = 0; g < CM; g++) {
        if (g > 0 && !full[g]) continue;
        const size_t idx = (size_t)row * ncols + cb[g];
        Vec<T, VW, true> xo, hv, ov;
        xo.load(X + idx);
        hv.load(hsrc + idx);
        if (a.accumulate) ov.load_rw(out + idx);
#pragma unroll
        for (int i = 0; i < VW; i++) {
          if (OS) own_s[((r * CM + g) * VW + i) * kBlkThreads + threadIdx.x] = xo.v[i];
          else own[OS ? 0 : r][g][i] = xo.v[i];
          double res = (double)acc[r][g][i] + __dmul_rn((double)hv.v[i] + hshift, (double)xo.v[i]);
          if (a.accumulate) res += (double)ov.v[i];
          ov.v[i] = (T)res;
        }
        ov.store(out + idx);
      }
    }
  }
  // transposed write-out: column c gets this thread's rows contiguous (index c * nrows + r), as
  // 16-byte accesses when the block is full and the thread's rows form whole 16-byte runs
  constexpr int RW = 16 / sizeof(T);
  constexpr bool kRuns = RPT % RW == 0;
  const bool vec_out = kRuns && nr == kBlkRows && (a.nrows % RW) == 0;
#pragma unroll
  for (int g = 0; g < CM; g++) {
    if (g > 0 && !full[g]) continue;
#pragma unroll
    for (int i = 0; i < VW; i++) {
      const size_t o = (size_t)(cb[g] + i) * a.nrows + r0 + rlo;
      if constexpr (kRuns) {
        if (vec_out) {
#pragma unroll
          for (int r = 0; r < RPT; r += RW) {
            Vec<T, RW, true> v;
            if (kAlpha) {
#pragma unroll
              for (int q = 0; q < RW; q++)
                v.v[q] = OS ? own_s[(((r + q) * CM + g) * VW + i) * kBlkThreads + threadIdx.x]
                            : own[OS ? 0 : r + q][g][i];
            } else {
              v.load_rw(out + o + r);
#pragma unroll
              for (int q = 0; q < RW; q++) v.v[q] += acc[r + q][g][i];
            }
            v.store(kAlpha ? XT + o + r : out + o + r);
          }
          continue;
        }
      }
#pragma unroll
      for (int r = 0; r < RPT; r++) {
        if (rlo + r < nr) {
          if (kAlpha) XT[o + r] = OS ? own_s[((r * CM + g) * VW + i) * kBlkThreads + threadIdx.x] : own[OS ? 0 : r][g][i];
          else out[o + r] += acc[r][g][i];
        }
      }
    }
  }
}

// The one-pass symmetric alpha pass with CM column groups per thread: each thread covers CM
// 16-byte groups of columns, TC * VW columns apart (so every load of a warp is one contiguous
// 512-byte run), and reuses each staged table entry -- its ket, value, and address arithmetic -- for
// all CM groups.  16-byte rows only (the caller falls back to sigma_block_kernel otherwise).  Same
// per-element arithmetic and order as sigma_block_kernel<kSym>.
template <typename T, int G, int M, int CM>
__global__ void __launch_bounds__(kBlkThreads, M)
    sigma_sym_cm_kernel(BlockArgs a, const T *__restrict__ X, T *__restrict__ out) {
  constexpr int VW = 16 / sizeof(T);
  constexpr int TC = kBlkThreads / G;
  constexpr int RPT = kBlkRows / G;
  constexpr int W = CM * TC * VW;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint32_t *sd_ket = reinterpret_cast<uint32_t *>(smem_raw);
  T *sd_val = reinterpret_cast<T *>(smem_raw + ((a.max_d * 4 + 15) & ~15u));
  unsigned char *sp = smem_raw + ((a.max_d * 4 + 15) & ~15u) + a.max_d * sizeof(T);
  sp = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(sp) + 15) & ~(uintptr_t)15);
  uint32_t *ss_ket = reinterpret_cast<uint32_t *>(sp);
  int32_t *ss_pair = reinterpret_cast<int32_t *>(sp + a.max_s * 4);
  double *ss_val = reinterpret_cast<double *>(sp + ((a.max_s * 8 + 15) & ~15u));

  const uint32_t nrb = (a.nrows + kBlkRows - 1) / kBlkRows;
  const uint32_t rb = blockIdx.x % nrb, slab = blockIdx.x / nrb;
  const uint32_t r0 = rb * kBlkRows;
  const uint32_t ncols = a.ncols;
  const int nr = (int)min((uint32_t)kBlkRows, a.nrows - r0);
  const int grp = threadIdx.x / TC;
  uint32_t cb[CM];
  bool full[CM];
#pragma unroll
  for (int g = 0; g < CM; g++) {
    cb[g] = slab * W + g * TC * VW + (threadIdx.x % TC) * VW;
    full[g] = cb[g] + VW <= ncols;  // ncols is a multiple of VW: a group is all in or all out
  }

  const uint32_t dlo = __ldg(&a.d_off[r0]), dhi = __ldg(&a.d_off[r0 + nr]);
  const uint32_t slo = __ldg(&a.s_off[r0]), shi = __ldg(&a.s_off[r0 + nr]);
  for (uint32_t e = dlo + threadIdx.x; e < dhi; e += blockDim.x) {
    sd_ket[e - dlo] = __ldg(&a.d_ket[e]);
    sd_val[e - dlo] = val_of<T>(a.d_val, a.d_valf, e);
  }
  for (uint32_t e = slo + threadIdx.x; e < shi; e += blockDim.x) {
    ss_ket[e - slo] = __ldg(&a.s_ket[e]);
    ss_pair[e - slo] = __ldg(&a.s_pair[e]);
    ss_val[e - slo] = (double)val_of<T>(a.s_val, a.s_valf, e);
  }
  __syncthreads();
  if (!full[0]) return;

  T acc[RPT][CM][VW];
#pragma unroll
  for (int r = 0; r < RPT; r++)
#pragma unroll
    for (int g = 0; g < CM; g++)
#pragma unroll
      for (int i = 0; i < VW; i++) acc[r][g][i] = T(0);
  const int rlo = grp * RPT;
#pragma unroll
  for (int r = 0; r < RPT; r++) {
    if (rlo + r >= nr) continue;
    const uint32_t row = r0 + rlo + r;
    const uint32_t d0 = __ldg(&a.d_off[row]) - dlo, d1 = __ldg(&a.d_off[row + 1]) - dlo;
#pragma unroll 4
    for (uint32_t e = d0; e < d1; e++) {
      const T v = sd_val[e];
      const T *xr = X + (size_t)sd_ket[e] * ncols;
#pragma unroll
      for (int g = 0; g < CM; g++) {
        if (g > 0 && !full[g]) continue;
        Vec<T, VW, true> x;
        x.load(xr + cb[g]);
#pragma unroll
        for (int i = 0; i < VW; i++) acc[r][g][i] = madd(acc[r][g][i], v, x.v[i]);
      }
    }
    const uint32_t s0 = __ldg(&a.s_off[row]) - slo, s1 = __ldg(&a.s_off[row + 1]) - slo;
    for (uint32_t e = s0; e < s1; e++) {
      const uint32_t ket = ss_ket[e];
      const double v = ss_val[e];
      const int32_t ps = ss_pair[e];
      const int pr = (ps > 0 ? ps : -ps) - 1;
      const double sg = ps > 0 ? 1.0 : -1.0;
      const double *vrow = a.vd + (size_t)pr * a.L;
      const T *xr = X + (size_t)ket * ncols;
      const double *jr = a.jtab ? a.jtab + (size_t)__ldg(&a.pmap[pr]) * ncols : nullptr;
#pragma unroll
      for (int g = 0; g < CM; g++) {
        if (g > 0 && !full[g]) continue;
        Vec<T, VW, true> xv;
        xv.load(xr + cb[g]);
        double o[VW];
        if (jr) {
#pragma unroll
          for (int i = 0; i < VW; i += 2) {
            const double2 jj = __ldg(reinterpret_cast<const double2 *>(jr + cb[g] + i));
            o[i] = jj.x;
            o[i + 1] = jj.y;
          }
        } else {
#pragma unroll
          for (int i = 0; i < VW; i++) {
            uint64_t occ = __ldg(&a.col_str[cb[g] + i]);
            o[i] = 0.0;
            while (occ) {
              o[i] += __ldg(&vrow[lowest_bit(occ)]);
              occ &= occ - 1;
            }
          }
        }
#pragma unroll
        for (int i = 0; i < VW; i++) acc[r][g][i] += (T)__dmul_rn(v + sg * o[i], (double)xv.v[i]);
      }
    }
    const T *hsrc = sizeof(T) == 8 ? reinterpret_cast<const T *>(a.hii) : reinterpret_cast<const T *>(a.hii32);
    const double hshift = sizeof(T) == 8 ? -a.core_shift : a.core_shift;
#pragma unroll
    for (int g = 0; g < CM; g++) {
      if (g > 0 && !full[g]) continue;
      const size_t idx = (size_t)row * ncols + cb[g];
      Vec<T, VW, true> xo, hv, ov;
      xo.load(X + idx);
      hv.load(hsrc + idx);
#pragma unroll
      for (int i = 0; i < VW; i++)
        ov.v[i] = (T)((double)acc[r][g][i] + 0.5 * __dmul_rn((double)hv.v[i] + hshift, (double)xo.v[i]));
      ov.store(out + idx);
    }
  }
}

}  // namespace

int reorder_sign_apply_f64(sbd_tpb_handle *h, const double *x, double *y) {
  reorder_sign_kernel_f64<<<h->num_sms * 8, 256, 0, h->stream>>>(
      h->d_apar, h->d_bstr, (uint32_t)h->bstr.size(), h->ndet(), x, y);
  TPB_LAUNCHED(h);
  return SBD_TPB_OK;
}

int reorder_sign_apply_f32(sbd_tpb_handle *h, const float *x, float *y) {
  reorder_sign_kernel_f32<<<h->num_sms * 8, 256, 0, h->stream>>>(
      h->d_apar, h->d_bstr, (uint32_t)h->bstr.size(), h->ndet(), x, y);
  TPB_LAUNCHED(h);
  return SBD_TPB_OK;
}

template <typename T, bool kAlpha, int G, int M, bool OS = false, bool kSym = false>
int launch_block_cfg(sbd_tpb_handle *h, const BlockArgs &ba, const T *X, T *out, T *XT) {
  constexpr int VW = 16 / sizeof(T);
  constexpr int W = (kBlkThreads / G) * VW;
  const size_t nrb = (ba.nrows + kBlkRows - 1) / kBlkRows, nslab = (ba.ncols + W - 1) / W;
  const size_t blocks = nrb * nslab;
  if (blocks > 0x7fffffffull) return fail(SBD_TPB_ERR_INVALID, "sigma: grid too large");
  const size_t smem = ((ba.max_d * 4 + 15) & ~(size_t)15) + (size_t)ba.max_d * sizeof(T) + 16 +
                      ((ba.max_s * 8 + 15) & ~(size_t)15) + (size_t)ba.max_s * 8 + 16 +
                      (OS ? (size_t)(kBlkRows / G) * VW * kBlkThreads * sizeof(T) + 16 : 0);
  if (smem > h->smem_optin) return fail(SBD_TPB_ERR_INVALID, "sigma: table block exceeds shared memory");
  // 16-byte column accesses need every row of X to start 16-byte aligned
  const bool vec = (ba.ncols % VW) == 0 && (reinterpret_cast<uintptr_t>(X) % 16) == 0 &&
                   (reinterpret_cast<uintptr_t>(out) % 16) == 0 &&
                   (!XT || (reinterpret_cast<uintptr_t>(XT) % 16) == 0);
  auto kern = vec ? sigma_block_kernel<T, kAlpha, true, G, M, OS, kSym>
                  : sigma_block_kernel<T, kAlpha, false, G, M, OS, kSym>;
  TPB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  kern<<<(unsigned)blocks, kBlkThreads, smem, h->stream>>>(ba, X, out, XT);
  TPB_LAUNCHED(h);
  return SBD_TPB_OK;
}

// sigma_pass_cm_kernel launch (16-byte rows, no alpha-single x beta-single terms)
template <typename T, bool kAlpha, int G, int M, int CM, bool OS = false>
int launch_pass_cm(sbd_tpb_handle *h, const BlockArgs &ba, const T *X, T *out, T *XT) {
  constexpr int VW = 16 / sizeof(T);
  constexpr int W = CM * (kBlkThreads / G) * VW;
  const size_t nrb = (ba.nrows + kBlkRows - 1) / kBlkRows, nslab = (ba.ncols + W - 1) / W;
  const size_t blocks = nrb * nslab;
  if (blocks > 0x7fffffffull) return fail(SBD_TPB_ERR_INVALID, "sigma: grid too large");
  const size_t smem = ((ba.max_d * 4 + 15) & ~(size_t)15) + (size_t)ba.max_d * sizeof(T) + 16 +
                      ((ba.max_s * 8 + 15) & ~(size_t)15) + (size_t)ba.max_s * 8 + 16 +
                      (OS ? (size_t)(kBlkRows / G) * CM * VW * kBlkThreads * sizeof(T) + 16 : 0);
  if (smem > h->smem_optin) return fail(SBD_TPB_ERR_INVALID, "sigma: table block exceeds shared memory");
  auto kern = sigma_pass_cm_kernel<T, kAlpha, G, M, CM, OS>;
  TPB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  kern<<<(unsigned)blocks, kBlkThreads, smem, h->stream>>>(ba, X, out, XT);
  TPB_LAUNCHED(h);
  return SBD_TPB_OK;
}

// Launch shapes of the general passes.  16-byte rows without the alpha-single x beta-single terms
// take sigma_pass_cm_kernel; from a sweep (CUDA events, ms at 4e8 / 1e8 determinants, row groups /
// CTAs per SM / column groups, "os": own values parked in shared memory), all giving the same bits:
// FP32 alpha 2/7/2/os 3.10 / 1.31, 2/8/1/os 3.05 / 1.39, 2/8/2 3.19 / 1.30, 2/6/2 3.25 / 1.29, 2/8/2/os
// 3.58 / 1.33; FP32 beta 2/8/2 2.78 / 1.18, 2/7/2 2.92 / 1.22, 2/6/2 3.09 / 1.27, 4/8/2 8.67 / 2.23;
// FP64 alpha 2/7/2 5.52 / 2.18, 2/8/2 5.79 / 2.27, 2/6/2 5.97 / 2.33; FP64 beta 2/7/2 5.24 / 2.12, 2/8/2
// 5.31 / 2.15, 2/6/2 5.63 / 2.25, 2/9/2 5.82 / 3.06 -- against sigma_block_kernel's 3.31 / 1.45,
// 3.35 / 1.36, 6.38 / 2.52 and 5.76 / 2.71.  Other rows take sigma_block_kernel: FP32 alpha one row
// group per thread below 10,000 CTAs (norb=12 FCI 0.84 -> 0.48 ms with two groups above), the values
// for C^T parked in shared memory above.
template <typename T, bool kAlpha>
int launch_block(sbd_tpb_handle *h, const BlockArgs &ba, const T *X, T *out, T *XT) {
  constexpr int VW = 16 / sizeof(T);
  const bool rows16 = (ba.ncols % VW) == 0 && reinterpret_cast<uintptr_t>(X) % 16 == 0 &&
                      reinterpret_cast<uintptr_t>(out) % 16 == 0 && (!XT || reinterpret_cast<uintptr_t>(XT) % 16 == 0);
  if (rows16 && !ba.do_ab) {
    if constexpr (sizeof(T) == 4 && kAlpha) return launch_pass_cm<T, true, 2, 7, 2, true>(h, ba, X, out, XT);
    else if constexpr (sizeof(T) == 4) return launch_pass_cm<T, false, 2, 8, 2>(h, ba, X, out, XT);
    else if constexpr (kAlpha) return launch_pass_cm<T, true, 2, 7, 2>(h, ba, X, out, XT);
    else return launch_pass_cm<T, false, 2, 7, 2>(h, ba, X, out, XT);
  }
  if constexpr (sizeof(T) == 4 && kAlpha) {
    const size_t blocks_g1 =
        ((ba.nrows + kBlkRows - 1) / kBlkRows) * ((ba.ncols + kBlkThreads * 4 - 1) / (kBlkThreads * 4));
    if (blocks_g1 >= 10000) return launch_block_cfg<T, kAlpha, 2, 8, true>(h, ba, X, out, XT);
    return launch_block_cfg<T, kAlpha, 2, 6>(h, ba, X, out, XT);
  } else if constexpr (kAlpha) {
    return launch_block_cfg<T, kAlpha, 2, 7>(h, ba, X, out, XT);
  } else if constexpr (sizeof(T) == 4) {
    return launch_block_cfg<T, kAlpha, 2, 8>(h, ba, X, out, XT);
  } else {
    return launch_block_cfg<T, kAlpha, 2, 9>(h, ba, X, out, XT);
  }
}

// sigma_sym_cm_kernel launch (16-byte rows only)
template <typename T, int G, int M, int CM>
int launch_sym_cm(sbd_tpb_handle *h, const BlockArgs &ba, const T *X, T *out) {
  constexpr int VW = 16 / sizeof(T);
  constexpr int W = CM * (kBlkThreads / G) * VW;
  if ((ba.ncols % VW) || (reinterpret_cast<uintptr_t>(X) % 16) || (reinterpret_cast<uintptr_t>(out) % 16))
    return fail(SBD_TPB_ERR_INVALID, "sigma: one-pass kernel needs 16-byte rows");
  const size_t nrb = (ba.nrows + kBlkRows - 1) / kBlkRows, nslab = (ba.ncols + W - 1) / W;
  const size_t blocks = nrb * nslab;
  if (blocks > 0x7fffffffull) return fail(SBD_TPB_ERR_INVALID, "sigma: grid too large");
  const size_t smem = ((ba.max_d * 4 + 15) & ~(size_t)15) + (size_t)ba.max_d * sizeof(T) + 16 +
                      ((ba.max_s * 8 + 15) & ~(size_t)15) + (size_t)ba.max_s * 8 + 16;
  if (smem > h->smem_optin) return fail(SBD_TPB_ERR_INVALID, "sigma: table block exceeds shared memory");
  auto kern = sigma_sym_cm_kernel<T, G, M, CM>;
  TPB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  kern<<<(unsigned)blocks, kBlkThreads, smem, h->stream>>>(ba, X, out);
  TPB_LAUNCHED(h);
  return SBD_TPB_OK;
}

// The symmetric alpha pass: no C^T and no values kept for it.  Launch shapes from sweeps (CUDA
// events, ms at 4e8 / 1e8 determinants), all giving the same bits.  With two column groups per
// thread (sigma_sym_cm_kernel, row groups / CTAs per SM / column groups): FP32 4/10/2 2.03 / 0.95,
// 2/8/2 2.09 / 0.99, 2/6/2 2.10 / 0.99, 4/8/2 2.14 / 0.97, 4/12/2 2.07 / 1.31, and one column
// group 2/8/1 2.19 / 1.01; FP64 2/8/2 3.77 / 1.75, 4/10/2 3.81 / 2.08, 2/6/2 4.04 / 1.82, 4/8/2
// 4.17 / 1.82, 2/8/1 4.17 / 2.13.  The general kernel's form (sigma_block_kernel<kSym>, kept for
// rows that are not 16-byte aligned) took FP32 2.78 / 1.22 and FP64 4.83 / 2.08 at its best shape.
template <typename T>
int launch_block_sym(sbd_tpb_handle *h, const BlockArgs &ba, const T *X, T *out) {
  const bool rows16 = (ba.ncols % (16 / sizeof(T))) == 0 && reinterpret_cast<uintptr_t>(X) % 16 == 0 &&
                      reinterpret_cast<uintptr_t>(out) % 16 == 0;
  if (!rows16) return launch_block_cfg<T, true, 2, 8, false, true>(h, ba, X, out, nullptr);
  if constexpr (sizeof(T) == 4) return launch_sym_cm<T, 4, 10, 2>(h, ba, X, out);
  else return launch_sym_cm<T, 2, 8, 2>(h, ba, X, out);
}

// Most entries of any kBlkRows-row block of a CSR table of n rows (shared-memory staging size).
int max_block_entries(const ExTable &t, size_t n, uint32_t *out) {
  *out = 0;
  if (n == 0) return SBD_TPB_OK;
  std::vector<uint32_t> off(n + 1);
  TPB_CUDA(cudaMemcpy(off.data(), t.off, sizeof(uint32_t) * (n + 1), cudaMemcpyDeviceToHost));
  uint32_t mx = 0;
  for (size_t r = 0; r < n; r += kBlkRows) mx = std::max(mx, off[std::min(n, r + kBlkRows)] - off[r]);
  *out = mx;
  return SBD_TPB_OK;
}

// The most table entries of any kBlkRows-row block of each table (the shared-memory staging of
// the sigma kernels), read back once per table build; blk_for records the tables they describe
// and is set only when all four were read.
int prepare_block_sizes(sbd_tpb_handle *h) {
  if (h->blk_for == (const void *)h->ta_d.ket) return SBD_TPB_OK;
  const size_t na = h->astr.size(), nb = h->bstr.size();
  uint32_t m[4];
  TPB_CHECK(max_block_entries(h->ta_d, na, &m[0]));
  TPB_CHECK(max_block_entries(h->ta_s, na, &m[1]));
  TPB_CHECK(max_block_entries(h->tb_d, nb, &m[2]));
  TPB_CHECK(max_block_entries(h->tb_s, nb, &m[3]));
  for (int i = 0; i < 4; i++) h->blk_max[i] = m[i];
  h->blk_for = h->ta_d.ket;
  return SBD_TPB_OK;
}

// Host-side facts about the tables that size the sigma launches: the per-block table sizes
// (prepare_block_sizes, done at table build) and, when want_ab_lists, the alpha rows and beta
// columns that have singles (the sparse alpha-beta launch).  Computed once per table build.
int prepare_sigma_meta(sbd_tpb_handle *h, bool want_ab_lists) {
  const size_t na = h->astr.size(), nb = h->bstr.size();
  TPB_CHECK(prepare_block_sizes(h));
  if (want_ab_lists && !h->d_ab_rows && na > 0 && nb > 0) {
    std::vector<uint32_t> ao(na + 1), bo(nb + 1), rows;
    TPB_CUDA(cudaMemcpy(ao.data(), h->ta_s.off, sizeof(uint32_t) * (na + 1), cudaMemcpyDeviceToHost));
    TPB_CUDA(cudaMemcpy(bo.data(), h->tb_s.off, sizeof(uint32_t) * (nb + 1), cudaMemcpyDeviceToHost));
    uint32_t kmax = 0;
    for (size_t i = 0; i < na; i++)
      if (ao[i + 1] > ao[i]) {
        rows.push_back((uint32_t)i);
        kmax = std::max(kmax, ao[i + 1] - ao[i]);
      }
    // rows with the most singles (the longest CTAs) first, so the grid does not end on a tail of
    // them; every CTA owns its sigma row, so the order changes no result
    std::stable_sort(rows.begin(), rows.end(), [&](uint32_t x, uint32_t y) {
      return ao[x + 1] - ao[x] > ao[y + 1] - ao[y];
    });
    // beta program: columns with singles and their entries, packed so a thread needs one load
    // per column and one per entry
    const size_t nnz = bo[nb];
    std::vector<uint32_t> bket(std::max<size_t>(1, nnz));
    std::vector<int32_t> bpair(std::max<size_t>(1, nnz));
    if (nnz) {
      TPB_CUDA(cudaMemcpy(bket.data(), h->tb_s.ket, sizeof(uint32_t) * nnz, cudaMemcpyDeviceToHost));
      TPB_CUDA(cudaMemcpy(bpair.data(), h->pb.s_pair, sizeof(int32_t) * nnz, cudaMemcpyDeviceToHost));
    }
    // columns ordered by their number of singles (most first, then by column), entries regrouped
    // in that order: the lanes of a warp take consecutive columns and loop over their singles, so
    // similar counts side by side keep the lanes busy (in column order ~30 % of the lane
    // iterations did work at norb=28-32, ~96 % in this order); each column's entries keep their
    // order, so the sums are unchanged
    std::vector<uint32_t> cols;
    for (size_t i = 0; i < nb; i++)
      if (bo[i + 1] > bo[i]) cols.push_back((uint32_t)i);
    std::stable_sort(cols.begin(), cols.end(), [&](uint32_t x, uint32_t y) {
      return bo[x + 1] - bo[x] > bo[y + 1] - bo[y];
    });
    // the distinct kets of the beta singles, and each entry's ket as its position among them
    std::vector<uint32_t> kets(bket.begin(), bket.begin() + nnz);
    std::sort(kets.begin(), kets.end());
    kets.erase(std::unique(kets.begin(), kets.end()), kets.end());
    std::vector<uint32_t> kpos(std::max<size_t>(1, nnz));
    for (size_t f = 0; f < nnz; f++)
      kpos[f] = (uint32_t)(std::lower_bound(kets.begin(), kets.end(), bket[f]) - kets.begin());
    // Ket ranges: the kernel stages, per group of alpha singles, their C rows restricted to one
    // range of the kets, and every group re-reads the part of the beta program for that range.
    // With dense beta singles (more than 4 entries per distinct ket: the program is then many
    // times the bytes of a staged row) and more singles per row than one group holds at four CTAs
    // per SM, the fewest ranges that let a group hold min(8, most singles of a row) singles at two
    // CTAs per SM in FP64 (FP32 then holds twice as many); else one range.  Targets of 12, 16 and 24
    // singles per group (more, shorter ranges) measured slower: norb=18 / 8.7e7 determinants FP64
    // 510 -> 520 / 563 / 699 ms, norb=24 / 3.0e7 189 -> 213 / 261 / 774 ms; targets of 4 and 6 were within
    // 1 % of 8 there (FP64), FP32 norb=24 105 / 113 against 114 ms.
    const size_t nk = kets.size(), L2 = (size_t)h->L * h->L;
    const size_t b4 = h->smem_optin / 4 - 1024, b2 = h->smem_optin / 2 - 1024;
    uint32_t nch = 1;
    const bool dense = nk > 0 && nnz > 4 * nk;
    if (dense && b4 / ((nk + L2) * sizeof(double)) < kmax) {
      const size_t want = std::min<size_t>(8, kmax);
      while (nch < 64 && b2 / (((nk + nch - 1) / nch + L2) * sizeof(double)) < want) nch++;
    }
    const uint32_t chunk = nk > 0 ? (uint32_t)((nk + nch - 1) / nch) : 1;
    // program: per range, per column (most singles first) its entries in that range, in table order
    std::vector<uint2> colp, bsp(std::max<size_t>(1, nnz));
    size_t w = 0;
    for (uint32_t m = 0; m < nch; m++) {
      for (const uint32_t c : cols) {
        colp.push_back(make_uint2(c, (uint32_t)w));
        for (uint32_t f = bo[c]; f < bo[c + 1]; f++)
          if (kpos[f] / chunk == m) bsp[w++] = make_uint2(kpos[f], (uint32_t)bpair[f]);
      }
      colp.push_back(make_uint2(0u, (uint32_t)w));
    }
    const size_t ncs = cols.size();
    if (kets.empty()) kets.push_back(0);
    TPB_CUDA(cudaMalloc(&h->d_ab_rows, sizeof(uint32_t) * std::max<size_t>(1, rows.size())));
    TPB_CUDA(cudaMalloc(&h->d_ab_colp, sizeof(uint2) * colp.size()));
    TPB_CUDA(cudaMalloc(&h->d_ab_bsp, sizeof(uint2) * bsp.size()));
    TPB_CUDA(cudaMalloc(&h->d_ab_kets, sizeof(uint32_t) * kets.size()));
    TPB_CUDA(cudaMemcpy(h->d_ab_kets, kets.data(), sizeof(uint32_t) * kets.size(), cudaMemcpyHostToDevice));
    h->ab_nkets = nnz ? (uint32_t)kets.size() : 0;
    if (!rows.empty())
      TPB_CUDA(cudaMemcpy(h->d_ab_rows, rows.data(), sizeof(uint32_t) * rows.size(), cudaMemcpyHostToDevice));
    TPB_CUDA(cudaMemcpy(h->d_ab_colp, colp.data(), sizeof(uint2) * colp.size(), cudaMemcpyHostToDevice));
    TPB_CUDA(cudaMemcpy(h->d_ab_bsp, bsp.data(), sizeof(uint2) * bsp.size(), cudaMemcpyHostToDevice));
    h->ab_nrows = (uint32_t)rows.size();
    h->ab_ncols = (uint32_t)ncs;
    h->ab_max_k = kmax;
    h->ab_nchunks = nch;
    h->ab_chunk = chunk;
    h->ab_dense = dense;
  }
  return SBD_TPB_OK;
}

template <typename T>
int launch_ab_sparse(sbd_tpb_handle *h, const T *C, T *sigma, double scale = 1.0, bool upper = false) {
  if (h->ab_nrows == 0 || h->ab_ncols == 0) return SBD_TPB_OK;
  AbSparseArgs a{};
  a.scale = scale;
  a.upper = upper ? 1 : 0;
  a.rows = h->d_ab_rows;
  a.colp = h->d_ab_colp;
  a.bsp = h->d_ab_bsp;
  a.kets = h->d_ab_kets;
  a.nk = h->ab_nkets;
  a.ncols_s = h->ab_ncols;
  a.nchunks = h->ab_nchunks;
  a.chunk = h->ab_chunk;
  a.as_off = h->ta_s.off;
  a.as_ket = h->ta_s.ket;
  a.as_pair = h->pa.s_pair;
  a.eri = h->d_eri;
  a.L2 = h->L * h->L;
  a.nb = (uint32_t)h->bstr.size();
  // one staged single = its C row over one ket range and its integral row; with a dense beta
  // program (each group re-reads its range's part) the largest group that leaves 2 CTAs per SM,
  // else groups sized for 4 CTAs per SM.  Measured, ab term ms at the previous one range and 4 CTAs
  // -> ranges and 2 CTAs: norb=18 / 8.7e7 determinants (51 singles per string) FP32 875 -> 310,
  // FP64 825 -> 517; norb=24 / 1.9e8 (63 per string) FP32 2915 -> 1167, FP64 5270 -> 2070;
  // norb=24 / 3.0e7 FP32 162 -> 117, FP64 322 -> 191.  Sparse singles (norb=28-32 selected sets)
  // keep one range and 4 CTAs per SM: 2 CTAs took them from 0.71 to 1.1-1.2 ms (FP32).
  const size_t per = ((size_t)a.chunk + a.L2) * sizeof(T);
  const size_t target = std::max<size_t>(per, h->smem_optin / (h->ab_dense ? 2 : 4) - 1024);
  if (per <= h->smem_optin) {
    a.group = (uint32_t)std::max<size_t>(1, std::min<size_t>(target / per, h->ab_max_k));
    const size_t smem = a.group * per;
    const auto kern = a.nchunks > 1 ? ab_sparse_kernel<T, true, true> : ab_sparse_kernel<T, true, false>;
    TPB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<h->ab_nrows, 256, smem, h->stream>>>(a, C, sigma);
  } else {
    a.group = h->ab_max_k;
    const auto kern = a.nchunks > 1 ? ab_sparse_kernel<T, false, true> : ab_sparse_kernel<T, false, false>;
    kern<<<h->ab_nrows, 256, 0, h->stream>>>(a, C, sigma);
  }
  TPB_LAUNCHED(h);
  return SBD_TPB_OK;
}

template <typename T>
int sigma_sep_shift(sbd_tpb_handle *h, const T *C, T *sigma, int accumulate, double shift) {
  const uint32_t na = (uint32_t)h->astr.size(), nb = (uint32_t)h->bstr.size();
  // dense alpha-beta path only where the contraction runs on the tensor cores (FP32 vectors): in
  // FP64 the shared-memory sparse kernel is faster even at full-CI connectivity (norb=12 FCI:
  // 1.5 ms against 3.4 ms for the CUDA-core gather/contract/scatter)
  const bool dense_ab = h->ab.enabled && sizeof(T) == 4 && h->ab.tc_ready;
  const size_t n = h->ndet();
  if (h->ct_bytes < n * sizeof(T)) {
    if (h->d_ct) cudaFree(h->d_ct);
    h->d_ct = nullptr;
    h->ct_bytes = 0;
    TPB_CUDA(cudaMalloc(&h->d_ct, n * sizeof(double)));
    h->ct_bytes = n * sizeof(double);
  }
  T *CT = reinterpret_cast<T *>(h->d_ct);
  TPB_CHECK(prepare_sigma_meta(h, !dense_ab));
  // per-pair Coulomb sums of the singles over the other spin's strings (built once per problem)
  TPB_CHECK(build_coulomb_table(h, h->pa, h->d_bstr, nb));
  TPB_CHECK(build_coulomb_table(h, h->pb, h->d_astr, na));

  BlockArgs ba{};
  ba.s_off = h->ta_s.off;
  ba.s_ket = h->ta_s.ket;
  ba.s_val = h->pa.s_val;
  ba.s_valf = h->pa.s_valf;
  ba.s_pair = h->pa.s_pair;
  ba.d_off = h->ta_d.off;
  ba.d_ket = h->ta_d.ket;
  ba.d_val = h->pa.d_val;
  ba.d_valf = h->pa.d_valf;
  ba.col_str = h->d_bstr;
  ba.jtab = h->pa.jtab;
  ba.pmap = h->pa.pmap;
  ba.vd = h->d_vd;
  ba.L = h->L;
  ba.nrows = na;
  ba.ncols = nb;
  ba.max_d = h->blk_max[0];
  ba.max_s = h->blk_max[1];
  ba.hii = h->d_hii;
  ba.hii32 = h->d_hii32;
  ba.core_shift = sizeof(T) == 8 ? shift : h->h00 - shift;
  ba.accumulate = accumulate;
  ba.do_ab = 0;  // alpha-beta terms: dense path or the sparse kernel below
  ba.bs_off = h->tb_s.off;
  ba.bs_ket = h->tb_s.ket;
  ba.bs_pair = h->pb.s_pair;
  ba.eri = h->d_eri;
  TPB_CUDA(cudaEventRecord(h->ev0, h->stream));
  TPB_CHECK((launch_block<T, true>(h, ba, C, sigma, CT)));
  TPB_CUDA(cudaEventRecord(h->ev_k[0], h->stream));

  BlockArgs bb{};
  bb.s_off = h->tb_s.off;
  bb.s_ket = h->tb_s.ket;
  bb.s_val = h->pb.s_val;
  bb.s_valf = h->pb.s_valf;
  bb.s_pair = h->pb.s_pair;
  bb.d_off = h->tb_d.off;
  bb.d_ket = h->tb_d.ket;
  bb.d_val = h->pb.d_val;
  bb.d_valf = h->pb.d_valf;
  bb.col_str = h->d_astr;
  bb.jtab = h->pb.jtab;
  bb.pmap = h->pb.pmap;
  bb.vd = h->d_vd;
  bb.L = h->L;
  bb.nrows = nb;
  bb.ncols = na;
  bb.max_d = h->blk_max[2];
  bb.max_s = h->blk_max[3];
  TPB_CHECK((launch_block<T, false>(h, bb, CT, sigma, nullptr)));
  TPB_CUDA(cudaEventRecord(h->ev_k[1], h->stream));
  if (dense_ab) {
    TPB_CHECK(ab_dense_apply<T>(h, C, sigma));
  } else {
    TPB_CHECK(launch_ab_sparse<T>(h, C, sigma));
  }
  TPB_CUDA(cudaEventRecord(h->ev_k[2], h->stream));
  h->sigma_kernels = 3;
  TPB_CUDA(cudaEventRecord(h->ev1, h->stream));
  return SBD_TPB_OK;
}

// sigma = (H - shift) C for an exchange-symmetric C (C = C^T, alpha strings = beta strings): the
// symmetric alpha pass writes B = (H_ii - shift) C / 2 + sum_Ja H_a(Ia, Ja) C[Ja, Ib], the
// alpha-beta term adds in at half weight (it is symmetric for a symmetric C), and sym_add forms
// sigma = B + B^T in place: the beta part of sigma is the transpose of the alpha part, the halves
// of the diagonal and alpha-beta terms add back.  One gathering pass instead of two and no C^T;
// sigma comes out exactly symmetric.  The result is sigma up to rounding only when C is
// symmetric; the caller guarantees that (Davidson with the exchange-symmetry projection).  With
// m > 0 the transpose-add also reduces S_k . sigma for the m vectors S (exactly symmetric too)
// into scalar slots slot.. (the Davidson step's new column of the projected matrix).
template <typename T>
int sigma_sep_sym(sbd_tpb_handle *h, const T *C, T *sigma, double shift, const T *const *S, int m,
                  int slot) {
  const uint32_t na = (uint32_t)h->astr.size(), nb = (uint32_t)h->bstr.size();
  if (na != nb || h->astr != h->bstr)
    return fail(SBD_TPB_ERR_STATE, "symmetric sigma needs identical alpha and beta strings");
  const bool dense_ab = h->ab.enabled && sizeof(T) == 4 && h->ab.tc_ready;
  TPB_CHECK(prepare_sigma_meta(h, !dense_ab));
  TPB_CHECK(build_coulomb_table(h, h->pa, h->d_bstr, nb));
  BlockArgs ba{};
  ba.s_off = h->ta_s.off;
  ba.s_ket = h->ta_s.ket;
  ba.s_val = h->pa.s_val;
  ba.s_valf = h->pa.s_valf;
  ba.s_pair = h->pa.s_pair;
  ba.d_off = h->ta_d.off;
  ba.d_ket = h->ta_d.ket;
  ba.d_val = h->pa.d_val;
  ba.d_valf = h->pa.d_valf;
  ba.col_str = h->d_bstr;
  ba.jtab = h->pa.jtab;
  ba.pmap = h->pa.pmap;
  ba.vd = h->d_vd;
  ba.L = h->L;
  ba.nrows = na;
  ba.ncols = nb;
  ba.max_d = h->blk_max[0];
  ba.max_s = h->blk_max[1];
  ba.hii = h->d_hii;
  ba.hii32 = h->d_hii32;
  ba.core_shift = sizeof(T) == 8 ? shift : h->h00 - shift;
  ba.accumulate = 0;
  ba.do_ab = 0;
  TPB_CUDA(cudaEventRecord(h->ev0, h->stream));
  TPB_CHECK(launch_block_sym<T>(h, ba, C, sigma));
  TPB_CUDA(cudaEventRecord(h->ev_k[0], h->stream));
  if (dense_ab) {
    TPB_CHECK(ab_dense_apply<T>(h, C, sigma, 0.5));
  } else {
    TPB_CHECK(launch_ab_sparse<T>(h, C, sigma, 1.0, true));
  }
  TPB_CUDA(cudaEventRecord(h->ev_k[1], h->stream));
  if (m > 0) TPB_CHECK(sym_add_dots<T>(h, sigma, S, m, slot));
  else TPB_CHECK(sym_add<T>(h, sigma));
  TPB_CUDA(cudaEventRecord(h->ev_k[2], h->stream));
  h->sigma_kernels = 3;
  TPB_CUDA(cudaEventRecord(h->ev1, h->stream));
  return SBD_TPB_OK;
}

template int sigma_sep_sym<double>(sbd_tpb_handle *, const double *, double *, double, const double *const *,
                                   int, int);
template int sigma_sep_sym<float>(sbd_tpb_handle *, const float *, float *, double, const float *const *, int,
                                  int);

// Same two passes with a caller-provided C^T buffer and the alpha-beta terms always evaluated by
// the direct loop of the alpha pass: needs no device memory beyond C, sigma and CT.
template <typename T>
int sigma_sep_given_ct(sbd_tpb_handle *h, const T *C, T *sigma, int accumulate, T *CT) {
  const uint32_t na = (uint32_t)h->astr.size(), nb = (uint32_t)h->bstr.size();
  TPB_CHECK(prepare_sigma_meta(h, false));
  BlockArgs ba{};
  ba.s_off = h->ta_s.off;
  ba.s_ket = h->ta_s.ket;
  ba.s_val = h->pa.s_val;
  ba.s_valf = h->pa.s_valf;
  ba.s_pair = h->pa.s_pair;
  ba.d_off = h->ta_d.off;
  ba.d_ket = h->ta_d.ket;
  ba.d_val = h->pa.d_val;
  ba.d_valf = h->pa.d_valf;
  ba.col_str = h->d_bstr;
  ba.vd = h->d_vd;
  ba.L = h->L;
  ba.nrows = na;
  ba.ncols = nb;
  ba.max_d = h->blk_max[0];
  ba.max_s = h->blk_max[1];
  ba.hii = h->d_hii;
  ba.hii32 = h->d_hii32;
  ba.core_shift = sizeof(T) == 8 ? 0.0 : h->h00;
  ba.accumulate = accumulate;
  ba.do_ab = 1;
  ba.bs_off = h->tb_s.off;
  ba.bs_ket = h->tb_s.ket;
  ba.bs_pair = h->pb.s_pair;
  ba.eri = h->d_eri;
  TPB_CUDA(cudaEventRecord(h->ev0, h->stream));
  TPB_CHECK((launch_block<T, true>(h, ba, C, sigma, CT)));
  TPB_CUDA(cudaEventRecord(h->ev_k[0], h->stream));
  BlockArgs bb{};
  bb.s_off = h->tb_s.off;
  bb.s_ket = h->tb_s.ket;
  bb.s_val = h->pb.s_val;
  bb.s_valf = h->pb.s_valf;
  bb.s_pair = h->pb.s_pair;
  bb.d_off = h->tb_d.off;
  bb.d_ket = h->tb_d.ket;
  bb.d_val = h->pb.d_val;
  bb.d_valf = h->pb.d_valf;
  bb.col_str = h->d_astr;
  bb.vd = h->d_vd;
  bb.L = h->L;
  bb.nrows = nb;
  bb.ncols = na;
  bb.max_d = h->blk_max[2];
  bb.max_s = h->blk_max[3];
  TPB_CHECK((launch_block<T, false>(h, bb, CT, sigma, nullptr)));
  TPB_CUDA(cudaEventRecord(h->ev_k[1], h->stream));
  h->sigma_kernels = 2;
  TPB_CUDA(cudaEventRecord(h->ev1, h->stream));
  return SBD_TPB_OK;
}

template int sigma_sep_given_ct<double>(sbd_tpb_handle *, const double *, double *, int, double *);
template int sigma_sep_given_ct<float>(sbd_tpb_handle *, const float *, float *, int, float *);

template <typename T>
int sigma_sep(sbd_tpb_handle *h, const T *C, T *sigma, int accumulate) {
  return sigma_sep_shift<T>(h, C, sigma, accumulate, 0.0);
}

template int sigma_sep<double>(sbd_tpb_handle *, const double *, double *, int);
template int sigma_sep<float>(sbd_tpb_handle *, const float *, float *, int);
template int sigma_sep_shift<double>(sbd_tpb_handle *, const double *, double *, int, double);
template int sigma_sep_shift<float>(sbd_tpb_handle *, const float *, float *, int, double);

}  // namespace sbdtpb
