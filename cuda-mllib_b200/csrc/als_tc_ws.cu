// Warp-specialised tensor-core half-step (sm_100a): gather, hermitian and solve
// of different rows overlap inside one persistent CTA per SM.
//
// Work: a host-planned list of items (rows, or chunks of rows too long for one
// CTA), largest first, dealt round-robin to the CTAs (LPT balance for
// power-law degrees). A split row's chunks accumulate partial A_u, b_u into
// global slots; the chunk that finishes last sums them in chunk order and
// solves the row.
//
//   warps 4NG,  three producers, taking stages of 64 ratings in turn: 16-byte
//   4NG+2, +3   cp.async copies of the rated factor rows (half a warp per row,
//               one 16-byte piece per lane) into a 128B-swizzled MN-major
//               tile, the swizzle computed in the destination address; rows
//               past the item's end are zero-filled. The lanes also write r_uk
//               into tile column c_r = ld (a pad column the copies never
//               touch). Completion reaches the MMA thread through
//               cp.async.mbarrier.arrive. Column indices and ratings arrive
//               DI - 1 owned stages ahead through a per-producer cp.async ring
//               in shared memory, item metadata 32 items at a time, so no
//               dependent global load is on the critical path.
//   warp 4NG+1  MMA issuer (one thread): per stage, tcgen05.mma kind::f16,
//               A = tile^T (M = 128), B = the first N = roundup16(max(NP,
//               c_r + 1)) tile columns, into TMEM accumulator r mod 4 for row
//               r; tcgen05.commit frees the stage and, after the item's last
//               stage, marks the accumulator full. D[:f, :f] = sum theta
//               theta^T, D[:f, c_r] = b_u; the other columns below c_r are
//               zero, rows >= f are ignored.
//   warps 0 ..  NG solver warpgroups (rows r = g mod NG to group g): read b_u
//   4NG-1       with tcgen05.ld (thread m <- TMEM lane m = row m of A_u) and
//               keep the accumulator for the whole solve: CG whose products
//               read A_u from TMEM (warm start optimally scaled; Cholesky
//               fallback), or the register-tile Cholesky + FP64-residual
//               refinement, each group on its own named barrier.
//
// Every mbarrier wait is bounded and gives up when another role aborted; a
// timeout sets the error word and all roles leave their loops.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <cstdlib>
#include <mutex>
#include <type_traits>
#include <vector>

#include "als_common.cuh"
#include "als_internal.h"
#include "als_tcgen05.cuh"

namespace als {

namespace ws {
// NG solver warpgroups (warps 0 .. 4 NG - 1), then producer 0, the MMA warp
// and producers 1 and 2. Registers per thread are capped by the busiest SM
// sub-partition: 168 with NG = 1 or 2 (three warps), 128 with NG = 3 (four).
template <int NG> __host__ __device__ constexpr int threads() { return 128 * NG + 128; }
template <int NG> __host__ __device__ constexpr int prod_warp() { return 4 * NG; }  // 4NG+2, 4NG+3 too
template <int NG> __host__ __device__ constexpr int mma_warp() { return 4 * NG + 1; }
constexpr int NS = 6;                             // shared-memory stages
constexpr int kMaxAcc = 4;                        // TMEM accumulators at most
constexpr int kMaxGroups = 3;                     // solver warpgroups per CTA at most
// Shape of an instance by its Cholesky tile extent FP (f <= FP): up to f = 112
// a stage holds tile columns 0-127 (two 64-column atoms: the factor row and
// the rating column c_r = ld <= 120) and four 128-column accumulators fill
// TMEM. Above (f <= 128, ld <= 136) a stage needs a third atom and the MMA's N
// reaches 144, so TMEM holds three accumulators of 160 columns; a 128-wide
// Cholesky tile would need 136 tiles for 128 threads, so rows CG cannot finish
// are handed to a post-pass of the one-CTA-per-row kernel.
// Ratings per stage: every shared-memory operation of the MMA thread (its
// barrier wait, the stage-info read, the commit) waits behind the MMAs it has
// queued, so each stage's bookkeeping leaves the tensor pipe idle for roughly
// the time of three to four 128 x 112 x 16 MMAs; 128-rating stages (eight MMAs
// a stage) halve that per rating. The wide shape's three atoms keep 64-rating
// stages so that six stages fit in shared memory.
template <int FP> struct Dims {
  static constexpr bool kWide = FP > 112;
  static constexpr int kKS = kWide ? 64 : 128;        // ratings per stage
  static constexpr int kAtom = (kKS / 8) * 1024;      // one 64-element MN atom of a stage
  static constexpr int kAtoms = kWide ? 3 : 2;
  static constexpr int kStageBytes = kAtoms * kAtom;
  static constexpr int kDI = kWide ? 8 : 5;           // index-ring slots (stages fetched ahead + 1)
  static constexpr int kRingSlot = 8 * kKS + 48;      // column indices, ratings, three int4 of header
  static constexpr int kAcc = kWide ? 3 : 4;          // row n -> accumulator n mod kAcc
  static constexpr int kBufCols = kWide ? 160 : 128;  // TMEM columns per accumulator
  static constexpr bool kChol = !kWide;               // the in-kernel Cholesky fallback
};
// Row hand-over: the solver warpgroups claim the CTA's rows in order from a
// shared counter, each taking the next row when it is free. (With a fixed
// assignment, row n to group n mod NG, a group's next row n + NG reuses the
// accumulator of row n + NG - kAcc, which another group may still hold.) Row
// n is posted in slot n mod kRowSlots, as that slot's (n / kRowSlots)-th
// barrier phase. An mbarrier parity wait tells only the current and the
// preceding phase apart, so no wait may name a phase two ahead of its
// barrier's:
//  - rows are claimed in order and a group claims a row only after taking
//    and finishing its previous one, so at most NG rows are claimed and not
//    yet taken: row n - kRowSlots has been taken before any group waits for
//    row n;
//  - a group waits for row n's accumulator (its (n / kAcc)-th fill) only
//    once fill n / kAcc - 1, by row n - kAcc, is complete: of the kAcc rows
//    n - kAcc .. n - 1 the other NG - 1 < kAcc groups hold at most NG - 1
//    unfinished, so one of them has been finished, its accumulator seen
//    full, and the MMA fills rows in order;
//  - a producer posting row r waits for the slot's previous row,
//    r - kRowSlots, to have been taken. When it posts row r it has finished
//    its previous stage, (first stage of r) - P with P producers, whose slot
//    wait means the MMA has issued stage (first stage of r) - P - NS and so
//    acquired the accumulator of its row R' >= r - P - NS; every row up to
//    R' - kAcc >= r - P - NS - kAcc >= r - 13 has then handed its
//    accumulator back, so it has been taken, and r - 2 kRowSlots (two slot
//    uses back) is among them.
constexpr int kRowSlots = 24;
__host__ __device__ constexpr int row_slot(long long n) { return (int)(n % kRowSlots); }
__host__ __device__ constexpr unsigned row_parity(long long n) {
  return (unsigned)(n / kRowSlots) & 1u;
}
constexpr int kTmemCols = 512;                    // allocated: all of TMEM
constexpr int kFullCount = 33;                    // 32 cp.async arrivals + the rating-store arrive
constexpr int kProducers = 3;                     // producer warps, taking stages in turn
// Stage info word, written by the stage's producer before it arrives on the
// stage's full barrier and read by the MMA thread in one load: accumulator
// (bits 0-1), MMAs of K = 16 (bits 2-5), first and last stage of the row
// (bits 6, 7); kInfoEnd marks the end of the CTA's stages.
constexpr uint32_t kInfoEnd = 1u << 31;
__host__ __device__ constexpr uint32_t stage_word(int acc, int kmma, int first, int last) {
  return (uint32_t)acc | ((uint32_t)kmma << 2) | ((uint32_t)first << 6) | ((uint32_t)last << 7);
}
static_assert(NS % kProducers == 0, "a stage slot always belongs to the same producer");
}  // namespace ws

struct WsGeom {
  int nj;  // 16-byte pieces per factor row (ld_src / 8, at most 17)
};

// Per solver warpgroup: the fallback Cholesky's tile when shared memory has
// room for it (else the tile lives in global scratch, plan.chol) and vectors,
// the CG broadcast vector and reduction slots.
template <int FP, int NP, int NG, bool SIN>
struct WsLayoutT {
  static constexpr int LDS = FP + 1;
  static constexpr bool kChol = ws::Dims<FP>::kChol;  // wide instances have no tile
  static_assert(!kChol || (size_t)FP * LDS <= (size_t)kCholFloats, "Cholesky tile fits its scratch");
  static constexpr bool kSInSmem = SIN && kChol;
  static constexpr size_t kS = kSInSmem ? (size_t)FP * LDS * 4 : 0;
  static constexpr size_t oDg = kS, oBv = oDg + FP * 4, oXv = oBv + FP * 4, oTmp = oXv + FP * 4;
  static constexpr size_t oPs = (oTmp + FP * 4 + 15) / 16 * 16;
  // CG broadcast vectors: two barrier phases x two vectors x one entry per
  // thread of the warpgroup (the TMEM-resident solver uses the first 128)
  static constexpr int kPs = 512;
  static_assert(NP <= 128, "the broadcast vector covers every accumulator column");
  static constexpr size_t oRed = oPs + kPs * 4;
  // 64 CG partial sums (two barrier phases of 32) + 64 refinement
  static constexpr size_t oRd = (oRed + 128 * 4 + 7) / 8 * 8;
  static constexpr size_t oMisc = oRd + (size_t)FP * 8;
  static constexpr size_t oCnt = oMisc + 16;  // six 64-bit counters of the group
  static constexpr size_t kSolver = (oCnt + 48 + 127) / 128 * 128;
  static constexpr size_t oSolver = (size_t)ws::NS * ws::Dims<FP>::kStageBytes;
  static constexpr size_t oCtrl = oSolver + NG * kSolver;
  // full, empty per stage; acc_full, acc_empty per accumulator (row n uses
  // accumulator n mod kAcc); row_full, row_empty per row slot; drain; one
  // spare (16-byte multiple)
  static constexpr size_t kBars = 8 * (2 * ws::NS + 2 * ws::kMaxAcc + 2 * ws::kRowSlots + 2);
  static constexpr size_t kCtrl = kBars + 16 * (ws::NS + ws::kRowSlots) + 16;
  static constexpr size_t oRing = oCtrl + kCtrl;  // 16-byte aligned
  static constexpr size_t kTotal =
      1024 + oRing + (size_t)ws::kProducers * ws::Dims<FP>::kDI * ws::Dims<FP>::kRingSlot;
  static_assert(kCtrl % 16 == 0 && ws::Dims<FP>::kRingSlot % 16 == 0, "ring alignment");
};

template <int FP, int NP, int NG>
using WsLayout = typename std::conditional<WsLayoutT<FP, NP, NG, true>::kTotal <= 232448,
                                           WsLayoutT<FP, NP, NG, true>,
                                           WsLayoutT<FP, NP, NG, false>>::type;

struct WsCtrl {
  uint64_t *full, *empty, *acc_full, *acc_empty, *row_full, *row_empty, *drain;
  uint32_t *stage_info;  // one info word per stage slot
  int4 *row_info;
  volatile int *misc;  // [0] TMEM base, [1] abort, [2] producer queue slot, [3] rows claimed
};

__device__ __forceinline__ void ws_abort(const RowsArgs &a, const WsCtrl &c) {
  atomicCAS(a.error, 0, 1);
  c.misc[1] = 1;
}

// ---------------------------------------------------------------------------
// producer warp
// ---------------------------------------------------------------------------
// No memory clobber: the copies are ordered by the mbarrier operations (all
// asm volatile) around them, and the column indices feeding a run of copies
// can be loaded ahead of it.
__device__ __forceinline__ void cp_async16_zfill(uint32_t dst, const void *src, uint32_t bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(bytes));
}
__device__ __forceinline__ void cp_async16_nc(uint32_t dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src));
}

__device__ __forceinline__ void mbar_arrive_cnt(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0], %1;" ::"r"(tc::smem_u32(bar)), "r"(count)
               : "memory");
}

// Work items are read a batch of 32 at a time (lane l holds the CTA's item
// 32 * batch + l) and handed out with shuffles, so the next item's metadata
// never waits on a load.
struct ItemBatch {
  int4 lo, hi;  // raw words of a WorkItem: {s, e}, {u, deg, part, heavy}
};

__device__ __forceinline__ ItemBatch load_batch(const WsPlan &p, long long bi, int lane) {
  const long long i = blockIdx.x + (bi * 32 + lane) * (long long)gridDim.x;
  // the item count of a plan built on the device is read from device memory
  const int nitems = p.nitems_dev ? *p.nitems_dev : p.nitems;
  ItemBatch b;
  if (i < nitems) {
    const int4 *q = reinterpret_cast<const int4 *>(p.items + i);
    b.lo = q[0];
    b.hi = q[1];
  } else {
    b.lo = make_int4(0, 0, 0, 0);
    b.hi = make_int4(-1, -1, -1, -1);
  }
  return b;
}

__device__ __forceinline__ void cp_async4(uint32_t dst, const void *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(dst), "l"(src) : "memory");
}

// Fetch cursor of a producer warp: walks the CTA's items stage by stage (the
// global stage sequence every producer sees alike) and copies the column
// indices and ratings of the stages it owns into its shared-memory ring with
// cp.async (one commit group per owned stage). Rows without ratings are
// finished by the cursor of producer 0 (x_u = 0).
template <typename LP, int KS>
struct FetchCursor {
  ItemBatch cb, nb;
  long long bi;
  int bpos;
  long long s, e, k0;
  int u, deg, part, heavy;
  int row;  // rows with ratings before the current item
  int gs;   // global index of the current stage
  bool owner;

  __device__ __forceinline__ void extract() {
    s = ((long long)__shfl_sync(0xffffffffu, cb.lo.y, bpos) << 32) |
        (unsigned)__shfl_sync(0xffffffffu, cb.lo.x, bpos);
    e = ((long long)__shfl_sync(0xffffffffu, cb.lo.w, bpos) << 32) |
        (unsigned)__shfl_sync(0xffffffffu, cb.lo.z, bpos);
    u = __shfl_sync(0xffffffffu, cb.hi.x, bpos);
    deg = __shfl_sync(0xffffffffu, cb.hi.y, bpos);
    part = __shfl_sync(0xffffffffu, cb.hi.z, bpos);
    heavy = __shfl_sync(0xffffffffu, cb.hi.w, bpos);
  }
  __device__ __forceinline__ void next_item(const WsPlan &p, int lane) {
    if (++bpos == 32) {
      cb = nb;
      ++bi;
      nb = load_batch(p, bi + 1, lane);
      bpos = 0;
    }
    extract();
  }
  // advance to the next item with ratings, finishing empty rows on the way
  __device__ __forceinline__ void settle(const RowsArgs &a, const WsPlan &p, int lane,
                                         unsigned long long &n_empty) {
    while (u >= 0 && e == s) {
      if (owner) {
        for (int i = lane; i < a.f; i += 32) {
          a.dst[(long long)u * a.ld_dst + i] = 0.f;
          if (a.dst_lp) reinterpret_cast<LP *>(a.dst_lp)[(long long)u * a.ld_dst_lp + i] = LP(0.f);
        }
        if (lane == 0) {
          if (a.row_flags) a.row_flags[u] = kRowEmpty;
          ++n_empty;
        }
      }
      next_item(p, lane);
    }
    k0 = s;
  }
  __device__ __forceinline__ void init(const RowsArgs &a, const WsPlan &p, int lane, bool own,
                                       unsigned long long &n_empty) {
    owner = own;
    bi = 0;
    bpos = 0;
    row = 0;
    gs = 0;
    cb = load_batch(p, 0, lane);
    nb = load_batch(p, 1, lane);
    extract();
    settle(a, p, lane, n_empty);
  }
  // move to the next global stage
  __device__ __forceinline__ void advance(const RowsArgs &a, const WsPlan &p, int lane,
                                          unsigned long long &n_empty) {
    if (u < 0) return;
    ++gs;
    k0 += KS;
    if (k0 >= e) {
      next_item(p, lane);
      settle(a, p, lane, n_empty);
      ++row;
    }
  }
  // copies of the current stage into ring slot rs, and its header: {u, deg,
  // part, heavy}, {kc, first, last, valid}, {row, stage}; past the end the
  // header is invalid and carries the number of rows and stages
  __device__ __forceinline__ void fetch(const RowsArgs &a, unsigned char *rs, int lane) {
    int4 *h = reinterpret_cast<int4 *>(rs + 8 * KS);
    if (u >= 0) {
      const int kc = (int)(e - k0 < KS ? e - k0 : KS);
      const uint32_t r0 = tc::smem_u32(rs);
#pragma unroll
      for (int j = 0; j < KS / 32; ++j) {
        const int k = lane + 32 * j;
        if (k < kc) {
          cp_async4(r0 + 4 * k, a.col + k0 + k);
          cp_async4(r0 + 4 * KS + 4 * k, a.val + k0 + k);
        }
      }
      if (lane == 0) {
        h[0] = make_int4(u, deg, part, heavy);
        h[1] = make_int4(kc, k0 == s ? 1 : 0, k0 + KS >= e ? 1 : 0, 1);
        h[2] = make_int4(row, gs, 0, 0);
      }
    } else if (lane == 0) {
      h[1] = make_int4(0, 0, 0, 0);
      h[2] = make_int4(row, gs, 0, 0);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  }
};

// One stage's factor rows: in each block of 64 rows, lanes 16h + j copy
// 16-byte piece j (< nj = ld / 8) of rows 32h .. 32h + 31 (< krows) into the
// 128B-swizzled MN-major tile (piece j of row k lands in atom j / 8, 8-row
// group k / 8, row k mod 8, 16-byte chunk (j mod 8) xor (k mod 8)). Rows at or
// past kc are zero-filled; a column index outside the factor matrix is clamped
// to its last row, so a malformed CSR gives wrong numbers but never reads
// outside the factors. The 32 column indices of a block are read first, so its
// copies issue back to back.
template <int KS>
__device__ __forceinline__ void gather_block(const RowsArgs &a, const WsPlan &plan, int j,
                                             int k0, const int *cols, int kc, int krows,
                                             uint32_t sa) {
  constexpr int kAtom = (KS / 8) * 1024;
  int ci[32];
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const int4 v = reinterpret_cast<const int4 *>(cols + k0)[q];
    ci[4 * q] = v.x;
    ci[4 * q + 1] = v.y;
    ci[4 * q + 2] = v.z;
    ci[4 * q + 3] = v.w;
  }
  const char *srcb = reinterpret_cast<const char *>(a.src) + 16 * j;
  const unsigned row_bytes = (unsigned)a.ld_src * 2u, last = (unsigned)plan.src_rows - 1u;
  const uint32_t dj = sa + (uint32_t)(j >> 3) * kAtom + (uint32_t)(k0 >> 3) * 1024;
  const uint32_t jx = (uint32_t)(j & 7) << 4;
  if (kc >= k0 + 32) {  // every row of this half carries a rating
#pragma unroll
    for (int i = 0; i < 32; ++i) {
      const unsigned c = min((unsigned)ci[i], last);
      const uint32_t dst = dj + (uint32_t)((i >> 3) * 1024 + (i & 7) * 128) + (jx ^ ((uint32_t)(i & 7) << 4));
      cp_async16_nc(dst, srcb + (size_t)c * row_bytes);
    }
  } else {
#pragma unroll
    for (int i = 0; i < 32; ++i) {
      const int k = k0 + i;
      if (k < krows) {
        const bool in = k < kc;
        const unsigned c = min((unsigned)ci[i], last);
        const char *src = in ? srcb + (size_t)c * row_bytes : srcb;
        const uint32_t dst = dj + (uint32_t)((i >> 3) * 1024 + (i & 7) * 128) + (jx ^ ((uint32_t)(i & 7) << 4));
        cp_async16_zfill(dst, src, in ? 16u : 0u);
      }
    }
  }
}

template <int KS>
__device__ __forceinline__ void gather_stage(const RowsArgs &a, const WsPlan &plan, int nj,
                                             const int *cols, int kc, int krows, uint32_t sa,
                                             int lane) {
  constexpr int kAtom = (KS / 8) * 1024;
  if (nj > 16) {
    // piece 16 (tile columns 128-135, atom 2, 16-byte chunk 0 xor (k mod 8)) of
    // rows lane, lane + 32, ..., for ranks f > 120
    const char *src16 = reinterpret_cast<const char *>(a.src) + 16 * 16;
    const unsigned row_bytes = (unsigned)a.ld_src * 2u, last = (unsigned)plan.src_rows - 1u;
    for (int k = lane; k < krows; k += 32) {
      const bool in = k < kc;
      const unsigned c = in ? min((unsigned)cols[k], last) : 0u;
      const uint32_t dst = sa + 2u * kAtom + (uint32_t)((k >> 3) * 1024 + (k & 7) * 128) +
                           ((uint32_t)(k & 7) << 4);
      cp_async16_zfill(dst, in ? src16 + (size_t)c * row_bytes : src16, in ? 16u : 0u);
    }
  }
  const int j = lane & 15;
  if (j >= nj) return;
#pragma unroll 1
  for (int k0 = (lane >> 4) * 32; k0 < krows; k0 += 64)
    gather_block<KS>(a, plan, j, k0, cols, kc, krows, sa);
}

// Producer k of ws::kProducers owns global stages k, k + kProducers, ...;
// stage t of the sequence goes to shared-memory stage t mod NS (the
// (t / NS)-th phase of its barriers), row r to row slot and accumulator
// r mod kAcc and to row slot row_slot(r), so the producers need no
// coordination beyond those barriers.
// The producer that owns the stage just past the last one writes the end
// markers.
template <int FP, typename LP, int NG>
__device__ void ws_produce(const RowsArgs &a, const WsPlan &plan, const WsGeom &g,
                           const WsCtrl &c, unsigned char *stages, unsigned char *ring, int k,
                           unsigned long long &n_empty_rows) {
  constexpr int P = ws::kProducers;
  using D = ws::Dims<FP>;
  constexpr int KS = D::kKS, DI = D::kDI;
  const int lane = threadIdx.x & 31;
  const uint32_t st0 = tc::smem_u32(stages);
  FetchCursor<LP, KS> fc;
  fc.init(a, plan, lane, k == 0, n_empty_rows);
  for (int i = 0; i < k; ++i) fc.advance(a, plan, lane, n_empty_rows);
  auto fetch_next = [&](long long t) {
    fc.fetch(a, ring + (int)(t % DI) * D::kRingSlot, lane);
    for (int i = 0; i < P; ++i) fc.advance(a, plan, lane, n_empty_rows);
  };
  for (int q = 0; q < DI - 1; ++q) fetch_next(q);
  bool ends = false;
  int end_rows = 0, end_stage = 0;
  for (long long t = 0;; ++t) {
    fetch_next(t + DI - 1);
    asm volatile("cp.async.wait_group %0;" ::"n"(DI - 1) : "memory");
    __syncwarp();
    const unsigned char *rs = ring + (int)(t % DI) * D::kRingSlot;
    const int4 *hd = reinterpret_cast<const int4 *>(rs + 8 * KS);
    const int4 h1 = hd[1], h2 = hd[2];
    if (__any_sync(0xffffffffu, h1.w == 0 || c.misc[1] != 0)) {  // warp-uniform exit
      ends = h1.w == 0 && c.misc[1] == 0 && h2.y == (int)(P * t + k);
      end_rows = h2.x;
      end_stage = h2.y;
      break;
    }
    const int kc = h1.x, first = h1.y, last = h1.z;
    const int st = (int)(P * t + k), slot = st % ws::NS;
    if (h2.y != st) {  // the cursors disagree: give up rather than mix up stages
      if (lane == 0) ws_abort(a, c);
      __syncwarp();
      break;
    }
    // every stage of row h2.x accumulates into accumulator h2.x mod kAcc, whichever
    // producer took the row's first stage
    const int acc = (int)((unsigned)h2.x % (unsigned)D::kAcc);
    if (first) {
      // the row's first stage also hands row h2.x to its solver group
      const int r = h2.x, rs2 = ws::row_slot(r);
      if (lane == 0) {
        bool okr = true;
        if (r >= ws::kRowSlots)  // the slot's previous row has been taken
          okr = tc::mbar_wait_or_abort(&c.row_empty[rs2], ws::row_parity(r - ws::kRowSlots),
                                       c.misc + 1);
        if (!okr) c.misc[1] = 1;
        c.row_info[rs2] = hd[0];
        tc::mbar_arrive(&c.row_full[rs2]);
      }
    }
    const int krows = (kc + 15) & ~15;
    bool okw = true;
    if (st >= ws::NS)
      okw = tc::mbar_wait_or_abort(&c.empty[slot], (unsigned)((st / ws::NS) - 1) & 1u, c.misc + 1);
    if (!__all_sync(0xffffffffu, okw)) { c.misc[1] = 1; break; }
    const uint32_t sa = st0 + (uint32_t)slot * D::kStageBytes;
    if (lane == 0) c.stage_info[slot] = ws::stage_word(acc, krows / 16, first, last);
    gather_stage<KS>(a, plan, g.nj, reinterpret_cast<const int *>(rs), kc, krows, sa, lane);
    // r_uk (0 past kc) into tile column c_r = 8 nj: atom c_r / 64, 16-byte
    // chunk ((c_r mod 64) / 8) xor (k mod 8), element 0; the chunk's other
    // elements stay zero
    const float *vr = reinterpret_cast<const float *>(rs + 4 * KS);
    const uint32_t rbase = sa + (uint32_t)(g.nj >> 3) * D::kAtom, rch = (uint32_t)(g.nj & 7);
    for (int kk = lane; kk < krows; kk += 32) {
      const uint16_t w = kk < kc ? tc::to_bits<LP>(vr[kk]) : (uint16_t)0;
      const uint32_t dst = rbase + (kk >> 3) * 1024 + (kk & 7) * 128 + ((rch ^ (uint32_t)(kk & 7)) << 4);
      asm volatile("st.shared.u16 [%0], %1;" ::"r"(dst), "h"(w));
    }
    tc::fence_proxy_async();             // the rating stores, for the tensor core
    tc::cp_async_arrive(&c.full[slot]);  // once this lane's copies have landed
    __syncwarp();
    if (lane == 0) tc::mbar_arrive(&c.full[slot]);  // releases the rating stores
  }
  asm volatile("cp.async.wait_all;" ::: "memory");  // no copy into the ring outlives the warp
  if (!ends) return;
  // end marker for the MMA thread at stage end_stage
  const int slot = end_stage % ws::NS;
  if (end_stage >= ws::NS)
    tc::mbar_wait_or_abort(&c.empty[slot], (unsigned)((end_stage / ws::NS) - 1) & 1u, c.misc + 1);
  if (lane == 0) {
    c.stage_info[slot] = ws::kInfoEnd;
    mbar_arrive_cnt(&c.full[slot], ws::kFullCount);
    // end markers: rows end_rows .. end_rows + NG - 1, the next row of each solver warpgroup
    for (int i = 0; i < NG; ++i) {
      const int r = end_rows + i, bb = ws::row_slot(r);
      if (r >= ws::kRowSlots)
        tc::mbar_wait_or_abort(&c.row_empty[bb], ws::row_parity(r - ws::kRowSlots), c.misc + 1);
      c.row_info[bb] = make_int4(-1, 0, 0, 0);
      tc::mbar_arrive(&c.row_full[bb]);
    }
  }
  __syncwarp();
}

// ---------------------------------------------------------------------------
// MMA issuer (one thread)
// ---------------------------------------------------------------------------
template <int FP>
__device__ void ws_mma(const RowsArgs &a, const WsCtrl &c, unsigned char *stages, uint32_t tmem,
                       uint32_t idesc, bool withhold_first) {
  // (test support: with withhold_first the issuer stops after the first item's
  // MMAs without marking its accumulator full, as an issuer that stalls would,
  // so the solvers' and producers' bounded waits run out)
  using D = ws::Dims<FP>;
  long long items_done = 0;
  // descriptors by addition: the start-address field (bits 0-13, address / 16)
  // of stage slot s, K step kk is that of slot 0 plus (s * stage + kk * 2 KB) / 16
  const uint64_t desc0 = tc::make_desc(tc::smem_u32(stages), D::kAtom, 1024);
  unsigned full_par = 0, acc_used = 0, acc_par = 0;
  int slot = 0;
  bool ok = true;
  for (;;) {
    ok = tc::mbar_wait_or_abort(&c.full[slot], (full_par >> slot) & 1, c.misc + 1);
    if (!ok) break;
    full_par ^= 1u << slot;
    const uint32_t info = *reinterpret_cast<const volatile uint32_t *>(&c.stage_info[slot]);
    if (info & ws::kInfoEnd) break;
    const int b = (int)(info & 3u), kmma = (int)((info >> 2) & 15u), first = (int)((info >> 6) & 1u),
              last = (int)((info >> 7) & 1u);
    // No proxy fence here: each producer lane fences its own generic stores of
    // the ratings before arriving, and the cp.async copies reach the barrier
    // only once they have landed (the pattern CUTLASS's sm100 cp.async
    // mainloop uses).
    if (first) {
      if (acc_used & (1u << b)) {
        ok = tc::mbar_wait_or_abort(&c.acc_empty[b], (acc_par >> b) & 1, c.misc + 1);
        if (!ok) break;
        acc_par ^= 1u << b;
      }
      acc_used |= 1u << b;
    }
    tc::tc_fence_after();
    const uint64_t ds = desc0 + (uint64_t)(((uint32_t)slot * D::kStageBytes) >> 4);
    const uint32_t td = tmem + (uint32_t)b * D::kBufCols;
    for (int kk = 0; kk < kmma; ++kk) {
      const uint64_t desc = ds + (uint64_t)(kk * (2048 >> 4));
      tc::mma_f16(td, desc, desc, idesc, (first && kk == 0) ? 0u : 1u);
    }
    tc::mma_commit(&c.empty[slot]);
    if (last) {
      if (withhold_first && items_done == 0) break;
      tc::mma_commit(&c.acc_full[b]);
      ++items_done;
    }
    slot = slot + 1 == ws::NS ? 0 : slot + 1;
  }
  if (!ok) ws_abort(a, c);
  tc::mma_commit(c.drain);  // every MMA issued so far has completed when this fires
  tc::mbar_wait(c.drain, 0);
}

// ---------------------------------------------------------------------------
// solver warpgroup
// ---------------------------------------------------------------------------
// Register-tile Cholesky of the system in S (identity padding beyond f),
// lambda * n_u added on the diagonal, triangular solves and the FP64-residual
// refinement; the solution lands in xv. Returns 0, 1 (not SPD: xv = 0) or 2
// (refined). Kept out of line so the CG loop is register-allocated on its own.
template <int FP>
__device__ __noinline__ int ws_cholesky(float *S, float *dg, float *bv, float *xv, float *tmp,
                                        double *rd, float *red, int *bad, int f, float reg,
                                        float refine_tol, const Bar &B) {
  constexpr int LDS = FP + 1, NTILES = (FP / 8) * (FP / 8 + 1) / 2;
  const int lt = B.tid;
  int ti = 0, tj = 0;
  const bool owner = lt < NTILES;
  if (owner) tile_of(lt, ti, tj);
  float acc[8][8];
  if (owner) {
#pragma unroll
    for (int r = 0; r < 8; ++r)
#pragma unroll
      for (int cc = 0; cc < 8; ++cc) {
        const int i = 8 * ti + r, j = 8 * tj + cc;
        float v = S[i * LDS + j];
        if (i == j && i < f) v += reg;
        acc[r][cc] = v;
      }
  }
  B.sync();
  if (owner && ti == tj) {
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      const int i = 8 * ti + r;
      dg[i] = acc[r][r];
      xv[i] = bv[i];
    }
  }
  const bool okc = tile_cholesky<FP, LDS, 128>(acc, ti, tj, owner, S, bad, B);
  if (!okc) {
    for (int i = lt; i < f; i += 128) xv[i] = 0.f;
    B.sync();
    return 1;
  }
  bool refined = false;
  solve_and_refine<FP, LDS, 128>(S, dg, bv, xv, rd, tmp, f, refine_tol, &refined, red, B);
  return refined ? 2 : 0;
}

// ---------------------------------------------------------------------------
// solver warpgroup, ranks up to 112 (system kept in TMEM)
// ---------------------------------------------------------------------------
// Row m of (D + diag I) times the broadcast vector v, with row m of D read
// from TMEM (lane m of accumulator tA) 32 columns at a time (64 per wait
// measured slower): the system stays
// in TMEM for the whole solve instead of occupying NP registers. Four
// independent FMA chains, carried two to an instruction by the packed FP32
// FMA of sm_100.
template <int NP>
__device__ __forceinline__ float matvec_tmem_np(uint32_t tA, const float *v, float diag, float vm) {
  float2 q01 = make_float2(diag * vm, 0.f), q23 = make_float2(0.f, 0.f);
#pragma unroll
  for (int c0 = 0; c0 < NP; c0 += 32) {
    float d[32];
    tc::tmem_ld32(tA + (uint32_t)c0, d);
#pragma unroll
    for (int k = 0; k < 32; k += 4) {
      if (c0 + k < NP) {
        const float4 p4 = *reinterpret_cast<const float4 *>(v + c0 + k);
        q01 = __ffma2_rn(make_float2(d[k], d[k + 1]), make_float2(p4.x, p4.y), q01);
        q23 = __ffma2_rn(make_float2(d[k + 2], d[k + 3]), make_float2(p4.z, p4.w), q23);
      }
    }
  }
  return (q01.x + q01.y) + (q23.x + q23.y);
}

// Sum of one per-thread value over the warpgroup: one barrier.
__device__ __forceinline__ float group_sum1(float a, float *red, int &slot, const Bar &B) {
  a = warp_sum(a);
  float *r = red + slot * 16;
  if ((B.tid & 31) == 0) r[B.tid >> 5] = a;
  B.sync();
  const float4 q = *reinterpret_cast<const float4 *>(r);
  slot ^= 1;
  return (q.x + q.y) + (q.z + q.w);
}

// Sum of two per-thread values over the warpgroup: one barrier. Within a warp
// the first shuffle level splits the work (lanes 0-15 keep summing a, lanes
// 16-31 b), so two sums cost five shuffles instead of ten.
__device__ __forceinline__ float2 group_sum2(float a, float b, float *red, int &slot,
                                             const Bar &B) {
  const int lane = B.tid & 31;
  const bool hi = lane & 16;
  float x = hi ? b : a;
  x += __shfl_xor_sync(0xffffffffu, hi ? a : b, 16);
#pragma unroll
  for (int o = 8; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  float *r = red + slot * 16;
  if ((lane & 15) == 0) r[(B.tid >> 5) * 2 + (lane >> 4)] = x;
  B.sync();
  float2 t = make_float2(0.f, 0.f);
#pragma unroll
  for (int w = 0; w < 4; ++w) {
    const float2 q = reinterpret_cast<const float2 *>(r)[w];
    t.x += q.x;
    t.y += q.y;
  }
  slot ^= 1;
  return t;
}

// Sum of four per-thread values over the warpgroup: one barrier. The first two
// shuffle levels split the four sums over lane quarters (six shuffles, not 20).
__device__ __forceinline__ float4 group_sum4(float4 v, float *red, int &slot, const Bar &B) {
  const int lane = B.tid & 31;
  const bool h16 = lane & 16, h8 = lane & 8;
  float x0 = h16 ? v.z : v.x, x1 = h16 ? v.w : v.y;
  x0 += __shfl_xor_sync(0xffffffffu, h16 ? v.x : v.z, 16);
  x1 += __shfl_xor_sync(0xffffffffu, h16 ? v.y : v.w, 16);
  float x = h8 ? x1 : x0;
  x += __shfl_xor_sync(0xffffffffu, h8 ? x0 : x1, 8);
#pragma unroll
  for (int o = 4; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  // lane 0: v.x, lane 8: v.y, lane 16: v.z, lane 24: v.w
  float *r = red + slot * 16;
  if ((lane & 7) == 0) r[(B.tid >> 5) * 4 + (lane >> 3)] = x;
  B.sync();
  float4 t = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
  for (int w = 0; w < 4; ++w) {
    const float4 q = reinterpret_cast<const float4 *>(r)[w];
    t.x += q.x; t.y += q.y; t.z += q.z; t.w += q.w;
  }
  slot ^= 1;
  return t;
}

// Solver warpgroup wg of NG claims the CTA's rows in order (the next one each
// time it is free). Row n arrives in row slot row_slot(n) and accumulator
// n mod kAcc (the (n / kAcc)-th phase of its barriers); the group keeps the
// accumulator until the row is solved: the CG matrix-vector products read A_u
// from TMEM.
template <int FP, int NP, typename LP, int NG>
__device__ void ws_solve(const RowsArgs &a, const WsPlan &plan, const TcSolve &sv,
                         const WsCtrl &c, unsigned char *mem, uint32_t tmem, int wg) {
  using L = WsLayout<FP, NP, NG>;
  constexpr int LDS = L::LDS, NTILES = (FP / 8) * (FP / 8 + 1) / 2;
  static_assert(NTILES <= 128, "one warpgroup holds at most 128 Cholesky tiles");
  static_assert(NP <= ws::Dims<FP>::kBufCols, "the system fits one accumulator");
  static_assert(!ws::Dims<FP>::kWide, "ranks up to 112");
  const int lt = threadIdx.x & 127, wl = (threadIdx.x >> 5) & 3;
  const Bar B{1 + wg, 128, lt};
  float *S = L::kSInSmem ? reinterpret_cast<float *>(mem)
                         : plan.chol + ((size_t)blockIdx.x * ws::kMaxGroups + wg) * kCholFloats;
  float *dg = reinterpret_cast<float *>(mem + L::oDg), *bv = reinterpret_cast<float *>(mem + L::oBv);
  float *xv = reinterpret_cast<float *>(mem + L::oXv), *tmp = reinterpret_cast<float *>(mem + L::oTmp);
  float *ps = reinterpret_cast<float *>(mem + L::oPs), *red = reinterpret_cast<float *>(mem + L::oRed);
  double *rd = reinterpret_cast<double *>(mem + L::oRd);
  int *bad = reinterpret_cast<int *>(mem + L::oMisc);
  const int f = a.f, m = lt;
  const bool live = m < f;
  ps[lt] = 0.f;  // L::kPs == 128 entries, one per thread
  B.sync();
  int rslot = 0;
  unsigned long long n_rows = 0, n_ref = 0, n_bad = 0, n_steps = 0, n_fb = 0, n_r0 = 0;
  const uint32_t tlane = tmem + ((uint32_t)(wl * 32) << 16);
  const uint32_t bcol = (uint32_t)(a.ld_src & ~15);
  const int bq = a.ld_src & 15;
  volatile int *claim = bad + 3;  // the row this group claimed last
  for (;;) {
    // the next row of the CTA; the barrier also ends every read of the
    // previous row's broadcast vector
    if (lt == 0) *claim = atomicAdd(const_cast<int *>(c.misc + 3), 1);
    B.sync();
    const long long n = *claim;
    const int rb = ws::row_slot(n), ab = (int)(n & (ws::Dims<FP>::kAcc - 1));
    const unsigned par = (unsigned)(n / ws::Dims<FP>::kAcc) & 1u;
    const uint32_t tA = tlane + (uint32_t)ab * ws::Dims<FP>::kBufCols;
    bool ok = tc::mbar_wait_or_abort(&c.row_full[rb], ws::row_parity(n), c.misc + 1);
    if (!B.all(ok)) { ws_abort(a, c); break; }
    const volatile int *vi = reinterpret_cast<volatile int *>(&c.row_info[rb]);
    const int4 info = make_int4(vi[0], vi[1], vi[2], vi[3]);
    tc::mbar_arrive(&c.row_empty[rb]);  // every thread, once it has read the slot
    if (info.x < 0) break;
    const int64_t u = info.x;
    const float reg = a.lambda * (float)info.y;
    // the warm start's load overlaps the wait for the accumulator
    float x = (live && sv.x0 && info.z < 0) ? sv.x0[u * sv.ld_x0 + m] : 0.f;
    ok = tc::mbar_wait_or_abort(&c.acc_full[ab], par, c.misc + 1);
    if (!B.all(ok)) { ws_abort(a, c); break; }
    tc::tc_fence_after();
    // b_u sits in column c_r = ld of D; rows >= f (no unknown) are ignored
    float bm = 0.f;
    {
      float v[16];
      tc::tmem_ld16(tA + bcol, v);
#pragma unroll
      for (int q = 0; q < 16; ++q)
        if (q == bq && live) bm = v[q];
    }
    if (info.z >= 0) {
      // A chunk of a split row: store the partial sums; the chunk that
      // finishes last adds all of them, in chunk order, into its own
      // accumulator and solves the row.
      float *P = plan.partial + ((size_t)info.z * 128 + m) * plan.part_ld;
#pragma unroll
      for (int c0 = 0; c0 < NP; c0 += 16) {
        float v[16];
        tc::tmem_ld16(tA + (uint32_t)c0, v);
#pragma unroll
        for (int q = 0; q < 16; q += 4)
          __stcg(reinterpret_cast<float4 *>(P + c0 + q),
                 live ? make_float4(v[q], v[q + 1], v[q + 2], v[q + 3]) : make_float4(0.f, 0.f, 0.f, 0.f));
      }
      __stcg(P + NP, bm);
      __threadfence();
      B.sync();
      if (lt == 0) {
        const unsigned done = atomicAdd(&plan.heavy_count[info.w], 1u) + 1;
        bad[1] = done == (unsigned)plan.heavy_nchunks[info.w] ? 1 : 0;
      }
      B.sync();
      const bool last = bad[1] != 0;
      B.sync();
      if (!last) {
        tc::tc_fence_before();
        tc::mbar_arrive(&c.acc_empty[ab]);
        continue;
      }
      __threadfence();
      const int base = plan.heavy_base[info.w], nch = plan.heavy_nchunks[info.w];
#pragma unroll
      for (int c0 = 0; c0 < NP; c0 += 16) {
        float v[16];
#pragma unroll
        for (int q = 0; q < 16; ++q) v[q] = 0.f;
        for (int ch = 0; ch < nch; ++ch) {
          const float *Q = plan.partial + ((size_t)(base + ch) * 128 + m) * plan.part_ld + c0;
#pragma unroll
          for (int q = 0; q < 16; q += 4) {
            const float4 w4 = __ldcg(reinterpret_cast<const float4 *>(Q + q));
            v[q] += w4.x;
            v[q + 1] += w4.y;
            v[q + 2] += w4.z;
            v[q + 3] += w4.w;
          }
        }
        tc::tmem_st16(tA + (uint32_t)c0, v);
      }
      bm = 0.f;
      for (int ch = 0; ch < nch; ++ch)
        bm += __ldcg(plan.partial + ((size_t)(base + ch) * 128 + m) * plan.part_ld + NP);
      if (lt == 0) plan.heavy_count[info.w] = 0;  // ready for the next half-step
      x = (live && sv.x0) ? sv.x0[u * sv.ld_x0 + m] : 0.f;
    }
    ++n_rows;
    uint32_t flags = 0;
    bool solved = false;
    float xm = 0.f;
    if (sv.solver == 1) {
      // Conjugate gradients on A_u = D + reg I, preconditioned by diag(A_u)
      // (Jacobi) unless disabled; three barriers per step.
      float dinv = live ? 1.f : 0.f;
      if (sv.jacobi) {
        float dm = 0.f;
#pragma unroll
        for (int c0 = 0; c0 < NP; c0 += 16) {
          float v[16];
          tc::tmem_ld16(tA + (uint32_t)c0, v);
#pragma unroll
          for (int q = 0; q < 16; ++q)
            if (c0 + q == m) dm = v[q];
        }
        if (live) dinv = 1.f / (dm + reg);
      }
      if (!isfinite(x)) x = 0.f;
      float r = bm;
      if (sv.x0) {
        // r = b - A x0. A learned start is first scaled optimally along its
        // own direction: alpha = x0.b / x0.A x0 minimises the A-norm error of
        // alpha * x0, so the start is never worse than zero in that norm. The
        // previous iterate is taken as it is (scaled, it needed more steps).
        // x0 is broadcast in the second quarter of ps, so the first can take
        // z while other threads still read x0.
        ps[128 + m] = x;
        B.sync();
        float q0 = matvec_tmem_np<NP>(tA, ps + 128, reg, x);
        if (!live) q0 = 0.f;
        if (sv.scale_x0) {
          const float2 xs = group_sum2(x * bm, x * q0, red, rslot, B);
          float sc = xs.x / xs.y;
          if (!(sc > 0.f) || !isfinite(sc)) sc = 0.f;
          x *= sc;
          r = bm - sc * q0;
        } else {
          r = bm - q0;
        }
      }
      if (!live) r = 0.f;
      float z = dinv * r;
      // Two barriers per step: z is broadcast through the same barrier that
      // sums r.z and r.r, and A p is carried by the recurrence
      // A p_k = A z_k + beta_k A p_{k-1} (p_k = z_k + beta_k p_{k-1}), so the
      // product is taken of z instead of p.
      ps[m] = z;
      const float4 t0 = group_sum4(make_float4(r * z, r * r, bm * bm, 0.f), red, rslot, B);
      float gamma = t0.x;
      const float bb = t0.z;
      const float target = sv.cg_tol2 * bb;
      if (lt == 0 && bb > 0.f) n_r0 += (unsigned long long)(1e6f * sqrtf(t0.y / bb));
      bool conv = t0.y <= target;
      int it = 0;
      float p = 0.f, w = 0.f, beta = 0.f;
      while (!conv && it < sv.cg_max_steps) {
        float az = matvec_tmem_np<NP>(tA, ps, reg, z);
        if (!live) az = 0.f;
        p = fmaf(beta, p, z);
        w = fmaf(beta, w, az);
        const float pq = group_sum1(p * w, red, rslot, B);
        if (!(pq > 0.f)) break;  // not positive definite along p: fall back
        const float alpha = __fdividef(gamma, pq);
        x = fmaf(alpha, p, x);
        r = fmaf(-alpha, w, r);
        z = dinv * r;
        ps[m] = z;  // read by the next product only after the barrier below
        const float2 t = group_sum2(r * z, r * r, red, rslot, B);
        ++it;
        conv = t.y <= target;
        beta = __fdividef(t.x, gamma);
        gamma = t.x;
      }
      if (lt == 0) n_steps += it;
      if (conv) {
        solved = true;
        xm = x;
      } else {
        flags |= kRowCgFallback;
        if (lt == 0) ++n_fb;
      }
    }
    if (!solved) {
      B.sync();  // the last reduction has been read: its slots and the tile are free
      // the system into shared memory for the register-tile Cholesky
#pragma unroll
      for (int c0 = 0; c0 < NP; c0 += 16) {
        float v[16];
        tc::tmem_ld16(tA + (uint32_t)c0, v);
        if (m < FP) {
#pragma unroll
          for (int q = 0; q < 16; ++q) {
            const int cc = c0 + q;
            if (cc < FP) S[m * LDS + cc] = (m < f && cc < f) ? v[q] : (m == cc ? 1.f : 0.f);
          }
        }
      }
      if (m < FP) {
        for (int cc = NP; cc < FP; ++cc) S[m * LDS + cc] = m == cc ? 1.f : 0.f;
        bv[m] = bm;
      }
      B.sync();
      const int res = ws_cholesky<FP>(S, dg, bv, xv, tmp, rd, red + 8, bad, f, reg, a.refine_tol, B);
      if (res == 1) {
        flags |= kRowNotSPD;
        if (lt == 0) ++n_bad;
      } else if (res == 2) {
        flags |= kRowRefinedF64;
        if (lt == 0) ++n_ref;
      }
      if (live) xm = xv[m];
      B.sync();
    }
    tc::tc_fence_before();
    tc::mbar_arrive(&c.acc_empty[ab]);  // the accumulator may be overwritten now
    if (live) {
      a.dst[u * a.ld_dst + m] = xm;
      if (a.dst_lp) reinterpret_cast<LP *>(a.dst_lp)[u * a.ld_dst_lp + m] = LP(xm);
    }
    if (a.row_flags && lt == 0) a.row_flags[u] = flags;
  }
  if (a.counters && lt == 0) {
    atomicAdd(&a.counters->rows, n_rows);
    if (n_ref) atomicAdd(&a.counters->refined, n_ref);
    if (n_bad) atomicAdd(&a.counters->not_spd, n_bad);
    if (n_steps) atomicAdd(&a.counters->cg_steps, n_steps);
    if (n_fb) atomicAdd(&a.counters->cg_fallback, n_fb);
    if (n_r0) atomicAdd(&a.counters->r0_micro, n_r0);
  }
}

// ---------------------------------------------------------------------------
// solver warpgroup, ranks above 112
// ---------------------------------------------------------------------------
// Row m of (D + diag I) times the broadcast vector v: four independent FMA
// chains over the columns in steps of eight, two lanes each (packed FP32
// FMA). matvec_reg takes row m of D from registers, matvec_tmem from TMEM lane
// m of accumulator tA; both do the same operations in the same order, so the
// two placements of the system give the same bits.
__device__ __forceinline__ void mv8(float2 (&q)[4], const float *A8, const float *v8) {
  const float4 a4 = *reinterpret_cast<const float4 *>(v8);
  const float4 b4 = *reinterpret_cast<const float4 *>(v8 + 4);
  q[0] = __ffma2_rn(make_float2(A8[0], A8[1]), make_float2(a4.x, a4.y), q[0]);
  q[1] = __ffma2_rn(make_float2(A8[2], A8[3]), make_float2(a4.z, a4.w), q[1]);
  q[2] = __ffma2_rn(make_float2(A8[4], A8[5]), make_float2(b4.x, b4.y), q[2]);
  q[3] = __ffma2_rn(make_float2(A8[6], A8[7]), make_float2(b4.z, b4.w), q[3]);
}
__device__ __forceinline__ float mv_total(const float2 (&q)[4]) {
  return ((q[0].x + q[0].y) + (q[1].x + q[1].y)) + ((q[2].x + q[2].y) + (q[3].x + q[3].y));
}

template <int KA>
__device__ __forceinline__ float matvec_reg(const float (&A)[KA], const float *v, float diag,
                                            float vm) {
  static_assert(KA % 8 == 0, "eight columns per step");
  float2 q[4] = {make_float2(diag * vm, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f),
                 make_float2(0.f, 0.f)};
#pragma unroll
  for (int k = 0; k < KA; k += 8) {
    // A compiler-only barrier every 32 columns keeps the vector's loads from
    // being hoisted all at once beside the row.
    if (k % 32 == 0 && k > 0) asm volatile("" ::: "memory");
    mv8(q, A + k, v + k);
  }
  return mv_total(q);
}

template <int KA>
__device__ __forceinline__ float matvec_tmem(uint32_t tA, const float *v, float diag, float vm) {
  static_assert(KA % 8 == 0, "eight columns per step");
  float2 q[4] = {make_float2(diag * vm, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f),
                 make_float2(0.f, 0.f)};
#pragma unroll
  for (int c0 = 0; c0 < KA; c0 += 32) {
    float d[32];
    if (KA - c0 > 16) {
      tc::tmem_ld32(tA + (uint32_t)c0, d);
    } else {
      float h[16];
      tc::tmem_ld16(tA + (uint32_t)c0, h);
#pragma unroll
      for (int k = 0; k < 16; ++k) d[k] = h[k];
    }
#pragma unroll
    for (int k = 0; k < 32; k += 8)
      if (c0 + k < KA) mv8(q, d + k, v + c0 + k);
  }
  return mv_total(q);
}

// The first half of a four-value warpgroup sum, split from its barrier so the
// barrier can also publish a broadcast vector: the warp's four partial sums
// (lane quarters split the shuffle tree: six shuffles for four sums) go to
// r[4 w .. 4 w + 3]. After the barrier, group_read4(r) gives the totals.
__device__ __forceinline__ void group_partial4(float4 v, float *r, int tid) {
  const int lane = tid & 31;
  const bool h16 = lane & 16, h8 = lane & 8;
  float x0 = h16 ? v.z : v.x, x1 = h16 ? v.w : v.y;
  x0 += __shfl_xor_sync(0xffffffffu, h16 ? v.x : v.z, 16);
  x1 += __shfl_xor_sync(0xffffffffu, h16 ? v.y : v.w, 16);
  float x = h8 ? x1 : x0;
  x += __shfl_xor_sync(0xffffffffu, h8 ? x0 : x1, 8);
#pragma unroll
  for (int o = 4; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  // lane 0: v.x, lane 8: v.y, lane 16: v.z, lane 24: v.w
  if ((lane & 7) == 0) r[(tid >> 5) * 4 + (lane >> 3)] = x;
}
// One and two values: the same split, with the shuffle trees of one value
// (five shuffles) and of two (lanes 0-15 keep a, 16-31 b: five shuffles).
__device__ __forceinline__ void group_partial1(float a, float *r, int tid) {
  a = warp_sum(a);
  if ((tid & 31) == 0) r[tid >> 5] = a;
}
__device__ __forceinline__ float group_read1(const float *r) {
  const float4 q = *reinterpret_cast<const float4 *>(r);
  return (q.x + q.y) + (q.z + q.w);
}
__device__ __forceinline__ void group_partial2(float a, float b, float *r, int tid) {
  const int lane = tid & 31;
  const bool hi = lane & 16;
  float x = hi ? b : a;
  x += __shfl_xor_sync(0xffffffffu, hi ? a : b, 16);
#pragma unroll
  for (int o = 8; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  if ((lane & 15) == 0) r[(tid >> 5) * 2 + (lane >> 4)] = x;
}
__device__ __forceinline__ float2 group_read2(const float *r) {
  float2 t = make_float2(0.f, 0.f);
#pragma unroll
  for (int w = 0; w < 4; ++w) {
    const float2 q = reinterpret_cast<const float2 *>(r)[w];
    t.x += q.x;
    t.y += q.y;
  }
  return t;
}
__device__ __forceinline__ float4 group_read4(const float *r) {
  float4 t = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
  for (int w = 0; w < 4; ++w) {
    const float4 q = reinterpret_cast<const float4 *>(r)[w];
    t.x += q.x; t.y += q.y; t.z += q.z; t.w += q.w;
  }
  return t;
}

// Columns [0, KA) of this thread's TMEM lane of accumulator tA into A (KA a
// multiple of 8, at most 128): every load issued before one wait. Each load
// fills a fixed-size array and all indices are constants, so everything
// stays in registers.
template <int KA>
__device__ __forceinline__ void tmem_row_to_regs(uint32_t tA, float (&A)[KA]) {
  static_assert(KA % 8 == 0 && KA <= 128, "row held in at most four 32-column loads");
  uint32_t r[4][32], t[16];
  constexpr int n32 = KA / 32, rem = KA - 32 * n32;  // rem in {0, 8, 16, 24}
#pragma unroll
  for (int b = 0; b < n32; ++b) tc::tmem_ld32_nowait(tA + 32 * b, r[b]);
  if constexpr (rem > 16) tc::tmem_ld32_nowait(tA + 32 * n32, r[n32 < 4 ? n32 : 0]);
  else if constexpr (rem > 0) tc::tmem_ld16_nowait(tA + 32 * n32, t);
  tc::tmem_wait_ld();
#pragma unroll
  for (int k = 0; k < KA; ++k) {
    uint32_t v = (k / 32 < n32 || rem > 16) ? r[k / 32][k % 32] : t[k % 32 < 16 ? k % 32 : 0];
    tc::tmem_launder(v);
    A[k] = __uint_as_float(v);
  }
}

// Where a solver warpgroup keeps the row's system while it solves it: in
// registers (thread m holds row m of A_u; the accumulator goes back to the MMA
// thread as soon as the row is copied out, so the next rows' hermitians
// accumulate while this one is solved), or in its TMEM accumulator (kept for
// the whole solve; for builds whose registers cannot hold a row).
template <int KA, bool REG>
struct RowSystem;
template <int KA>
struct RowSystem<KA, true> {
  float A[KA];
  __device__ __forceinline__ float mv(const float *v, float diag, float vm) const {
    return matvec_reg<KA>(A, v, diag, vm);
  }
  __device__ __forceinline__ void load(uint32_t tA) { tmem_row_to_regs<KA>(tA, A); }
  __device__ __forceinline__ void clear() {
#pragma unroll
    for (int k = 0; k < KA; ++k) A[k] = 0.f;
  }
  // the row into a row of the Cholesky tile (columns [0, KA)) when `write`
  __device__ __forceinline__ void store(float *Sr, bool write) const {
    if (!write) return;
#pragma unroll
    for (int k = 0; k < KA; ++k) Sr[k] = A[k];
  }
  // add a partial sum (a split row's chunk slot) into the row
  __device__ __forceinline__ void add(const float *Q) {
#pragma unroll
    for (int c0 = 0; c0 < KA; c0 += 4) {
      const float4 w4 = __ldcg(reinterpret_cast<const float4 *>(Q + c0));
      A[c0] += w4.x; A[c0 + 1] += w4.y; A[c0 + 2] += w4.z; A[c0 + 3] += w4.w;
    }
  }
  __device__ __forceinline__ void save_partial(float *P, bool live, uint32_t) const {
#pragma unroll
    for (int c0 = 0; c0 < KA; c0 += 4)
      __stcg(reinterpret_cast<float4 *>(P + c0),
             live ? make_float4(A[c0], A[c0 + 1], A[c0 + 2], A[c0 + 3]) : make_float4(0.f, 0.f, 0.f, 0.f));
  }
};
template <int KA>
struct RowSystem<KA, false> {
  uint32_t tA;
  __device__ __forceinline__ float mv(const float *v, float diag, float vm) const {
    return matvec_tmem<KA>(tA, v, diag, vm);
  }
  __device__ __forceinline__ void load(uint32_t t) { tA = t; }
  // Every thread of the warp must call this (the TMEM loads are
  // warp-collective); only threads with `write` store.
  __device__ __forceinline__ void store(float *Sr, bool write) const {
#pragma unroll
    for (int c0 = 0; c0 < KA; c0 += 16) {
      float v[16];
      tc::tmem_ld16(tA + (uint32_t)c0, v);
      if (write) {
#pragma unroll
        for (int q = 0; q < 16; ++q)
          if (c0 + q < KA) Sr[c0 + q] = v[q];
      }
    }
  }
  __device__ __forceinline__ void save_partial(float *P, bool live, uint32_t) const {
#pragma unroll
    for (int c0 = 0; c0 < KA; c0 += 16) {
      float v[16];
      tc::tmem_ld16(tA + (uint32_t)c0, v);
#pragma unroll
      for (int q = 0; q < 16; q += 4)
        if (c0 + q < KA)
          __stcg(reinterpret_cast<float4 *>(P + c0 + q),
                 live ? make_float4(v[q], v[q + 1], v[q + 2], v[q + 3]) : make_float4(0.f, 0.f, 0.f, 0.f));
    }
  }
  // the sum of a split row's chunk slots into the accumulator, in chunk order
  __device__ __forceinline__ void sum_partials(const float *partial, int base, int nch, int m,
                                               int part_ld) {
#pragma unroll
    for (int c0 = 0; c0 < KA; c0 += 16) {
      float v[16];
#pragma unroll
      for (int q = 0; q < 16; ++q) v[q] = 0.f;
      for (int ch = 0; ch < nch; ++ch) {
        const float *Q = partial + ((size_t)(base + ch) * 128 + m) * part_ld + c0;
#pragma unroll
        for (int q = 0; q < 16; q += 4) {
          if (c0 + q < KA) {
            const float4 w4 = __ldcg(reinterpret_cast<const float4 *>(Q + q));
            v[q] += w4.x; v[q + 1] += w4.y; v[q + 2] += w4.z; v[q + 3] += w4.w;
          }
        }
      }
      tc::tmem_st16(tA + (uint32_t)c0, v);
    }
  }
};

// Solver warpgroup wg of NG claims the CTA's rows in order (the next one each
// time it is free). Row n arrives in row slot row_slot(n) and accumulator
// n mod kAcc (the (n / kAcc)-th phase of its barriers). CG (optionally Jacobi-preconditioned)
// from the warm start scaled optimally along itself, to relative residual
// cg_tol in at most cg_max_steps steps; a reduction is written as partial sums
// before its barrier and read after it, and the barriers that publish the
// warm start and the search direction are the ones the group needs anyway (the
// accumulator vote, and the reduction of r.z and r.r). Rows CG does not
// finish, or along whose search direction A is not positive, are solved by the
// register-tile Cholesky with FP64-residual refinement; so is every row when
// sv.solver == 0.
template <int FP, int NP, typename LP, int NG, bool REG>
__device__ void ws_solve_wide(const RowsArgs &a, const WsPlan &plan, const TcSolve &sv,
                         const WsCtrl &c, unsigned char *mem, uint32_t tmem, int wg) {
  using L = WsLayout<FP, NP, NG>;
  constexpr int LDS = L::LDS, NTILES = (FP / 8) * (FP / 8 + 1) / 2;
  static_assert(!L::kChol || NTILES <= 128, "one warpgroup holds at most 128 Cholesky tiles");
  using D = ws::Dims<FP>;
  static_assert(NP <= D::kBufCols, "the system fits one accumulator");
  // columns of the system per thread: f <= min(NP, FP); the rest of the
  // accumulator is padding (and the b_u column)
  constexpr int KA = NP < FP ? NP : FP;
  const int lt = threadIdx.x & 127, wl = (threadIdx.x >> 5) & 3;
  const Bar B{1 + wg, 128, lt};
  float *S = L::kSInSmem ? reinterpret_cast<float *>(mem)
                         : plan.chol + ((size_t)blockIdx.x * ws::kMaxGroups + wg) * kCholFloats;
  float *dg = reinterpret_cast<float *>(mem + L::oDg), *bv = reinterpret_cast<float *>(mem + L::oBv);
  float *xv = reinterpret_cast<float *>(mem + L::oXv), *tmp = reinterpret_cast<float *>(mem + L::oTmp);
  float *pv = reinterpret_cast<float *>(mem + L::oPs), *red = reinterpret_cast<float *>(mem + L::oRed);
  double *rd = reinterpret_cast<double *>(mem + L::oRd);
  int *bad = reinterpret_cast<int *>(mem + L::oMisc);
  const int f = a.f, m = lt;
  const bool live = m < f;
  for (int i = lt; i < L::kPs; i += 128) pv[i] = 0.f;
  B.sync();
  // Phase of the barriers that publish vectors or partial sums: the k-th such
  // barrier of the group uses buffer k mod 2 (vectors pv[256 (k mod 2) ...],
  // partials red[32 (k mod 2) ...]). A buffer is written again only two
  // barriers later, when every thread has finished reading it.
  int ph = 0;
  auto vbuf = [&](int k) { return pv + (ph & 1) * 256 + k * 128; };
  auto rbuf = [&]() { return red + (ph & 1) * 32; };
  // counters of the group, kept by thread 0 in shared memory (not registers)
  unsigned long long *cnt = reinterpret_cast<unsigned long long *>(mem + L::oCnt);
  if (lt == 0)
    for (int k = 0; k < 6; ++k) cnt[k] = 0;
  const uint32_t tlane = tmem + ((uint32_t)(wl * 32) << 16);
  const uint32_t bcol = (uint32_t)(a.ld_src & ~15);
  const int bq = a.ld_src & 15;
  const bool cg = sv.solver == 1;
  volatile int *claim = bad + 3;  // the row this group claimed last
  for (;;) {
    // the next row of the CTA
    if (lt == 0) *claim = atomicAdd(const_cast<int *>(c.misc + 3), 1);
    B.sync();
    const long long n = *claim;
    const int rb = ws::row_slot(n);
    const int ab = (int)((unsigned long long)n % (unsigned)D::kAcc);
    const unsigned par = (unsigned)((unsigned long long)n / (unsigned)D::kAcc) & 1u;
    const uint32_t tA = tlane + (uint32_t)ab * D::kBufCols;
    bool ok = tc::mbar_wait_or_abort(&c.row_full[rb], ws::row_parity(n), c.misc + 1);
    int4 info = make_int4(-1, 0, 0, 0);
    if (ok) {
      const volatile int *vi = reinterpret_cast<volatile int *>(&c.row_info[rb]);
      info = make_int4(vi[0], vi[1], vi[2], vi[3]);
      tc::mbar_arrive(&c.row_empty[rb]);  // every thread, once it has read the slot
    }
    if (!B.all(ok)) { ws_abort(a, c); break; }
    if (info.x < 0) break;
    const int64_t u = info.x;
    const float reg = a.lambda * (float)info.y;
    // the warm start's load overlaps the wait for the accumulator, and (for a
    // whole row) it is published with the accumulator vote
    float x = (live && sv.x0 && info.z < 0) ? sv.x0[u * sv.ld_x0 + m] : 0.f;
    if (!isfinite(x)) x = 0.f;
    if (cg && info.z < 0) vbuf(0)[m] = x;
    ok = tc::mbar_wait_or_abort(&c.acc_full[ab], par, c.misc + 1);
    if (!B.all(ok)) { ws_abort(a, c); break; }
    if (cg && info.z < 0) ++ph;
    tc::tc_fence_after();
    RowSystem<KA, REG> sys;
    float bm;
    {
      float b16[16];
      tc::tmem_ld16(tA + bcol, b16);  // b_u sits in column c_r = ld of D
      bm = 0.f;
#pragma unroll
      for (int q = 0; q < 16; ++q)
        if (q == bq) bm = b16[q];
    }
    sys.load(tA);
    if constexpr (REG) {
      // the accumulator may be overwritten now
      tc::tc_fence_before();
      tc::mbar_arrive(&c.acc_empty[ab]);
    }
    if (info.z >= 0) {
      // A chunk of a split row: store the partial sums; the chunk that
      // finishes last adds all of them, in chunk order, and solves the row.
      float *P = plan.partial + ((size_t)info.z * 128 + m) * plan.part_ld;
      sys.save_partial(P, live, 0);
      __stcg(P + NP, live ? bm : 0.f);
      __threadfence();
      B.sync();
      if (lt == 0) {
        const unsigned done = atomicAdd(&plan.heavy_count[info.w], 1u) + 1;
        bad[1] = done == (unsigned)plan.heavy_nchunks[info.w] ? 1 : 0;
      }
      B.sync();
      const bool last = bad[1] != 0;
      B.sync();
      if (!last) {
        if constexpr (!REG) {
          tc::tc_fence_before();
          tc::mbar_arrive(&c.acc_empty[ab]);
        }
        continue;
      }
      __threadfence();
      const int base = plan.heavy_base[info.w], nch = plan.heavy_nchunks[info.w];
      if constexpr (REG) {
        sys.clear();
        for (int ch = 0; ch < nch; ++ch)
          sys.add(plan.partial + ((size_t)(base + ch) * 128 + m) * plan.part_ld);
      } else {
        sys.sum_partials(plan.partial, base, nch, m, plan.part_ld);
      }
      bm = 0.f;
      for (int ch = 0; ch < nch; ++ch)
        bm += __ldcg(plan.partial + ((size_t)(base + ch) * 128 + m) * plan.part_ld + NP);
      if (lt == 0) plan.heavy_count[info.w] = 0;  // ready for the next half-step
      x = (live && sv.x0) ? sv.x0[u * sv.ld_x0 + m] : 0.f;
      if (!isfinite(x)) x = 0.f;
      if (cg) {
        vbuf(0)[m] = x;
        B.sync();
        ++ph;
      }
    }
    // Rows past f carry no unknowns (row c_r of D holds b_u^T): a padding
    // thread's values are cleared, with one predicate per thread. Columns past
    // f need no clearing: they meet broadcast entries that are zero (every
    // published vector is zero past f), and the Cholesky tile is patched below.
    if constexpr (REG) {
      if (!live) sys.clear();
    }
    if (!live) bm = 0.f;
    uint32_t flags = 0;
    bool solved = false;
    float xm = 0.f;
    if (cg) {
      float dinv = live ? 1.f : 0.f;
      if (L::kChol && sv.jacobi) {  // (wide instances are not launched with Jacobi)
        // the diagonal entry A[m][m] sits at a thread-dependent column: go
        // through the (still unused) Cholesky tile for it (every thread calls
        // store: its TMEM loads are warp-collective)
        sys.store(S + (m < FP ? m : 0) * LDS, m < FP);
        __syncwarp();
        if (live) dinv = 1.f / (S[m * LDS + m] + reg);
      }
      float r = bm;
      if (sv.x0) {
        // r = b - A x0. A learned start is first scaled optimally along its
        // own direction: alpha = x0.b / x0.A x0 minimises the A-norm error of
        // alpha * x0, so the start is never worse than zero in that norm; the
        // previous iterate is taken as it is. x0 was published with the
        // accumulator vote (or after the split row's sums).
        float q0 = sys.mv(pv + ((ph - 1) & 1) * 256, reg, x);
        if (!live) q0 = 0.f;
        if (sv.scale_x0) {
          group_partial2(x * bm, x * q0, rbuf(), lt);
          B.sync();
          const float2 xs = group_read2(rbuf());
          ++ph;
          float sc = xs.x / xs.y;
          if (!(sc > 0.f) || !isfinite(sc)) sc = 0.f;
          x *= sc;
          r = bm - sc * q0;
        } else {
          r = bm - q0;
        }
      }
      if (!live) r = 0.f;
      float z = dinv * r;
      // z is broadcast through the barrier that sums r.z, r.r and b.b
      vbuf(0)[m] = z;
      group_partial4(make_float4(r * z, r * r, bm * bm, 0.f), rbuf(), lt);
      B.sync();
      const float4 t0 = group_read4(rbuf());
      const float *vz = vbuf(0);
      ++ph;
      float gamma = t0.x;
      const float bb = t0.z, target = sv.cg_tol2 * bb;
      if (lt == 0 && bb > 0.f) cnt[5] += (unsigned long long)(1e6f * sqrtf(t0.y / bb));
      bool conv = t0.y <= target;
      int it = 0;
      float p = 0.f, w = 0.f, beta = 0.f;
      // Conjugate gradients, two barriers a step: A p is carried by the
      // recurrence A p_k = A z_k + beta_k A p_{k-1} (p_k = z_k + beta_k p_{k-1}),
      // so the product is taken of z, which is broadcast through the same
      // barrier that sums r.z and r.r.
      while (!conv && it < sv.cg_max_steps) {
        float az = sys.mv(vz, reg, z);
        if (!live) az = 0.f;
        p = fmaf(beta, p, z);
        w = fmaf(beta, w, az);
        group_partial1(p * w, rbuf(), lt);
        B.sync();
        const float pq = group_read1(rbuf());
        ++ph;
        if (!(pq > 0.f)) break;  // not positive definite along p: fall back
        const float alpha = __fdividef(gamma, pq);
        x = fmaf(alpha, p, x);
        r = fmaf(-alpha, w, r);
        z = dinv * r;
        vbuf(0)[m] = z;
        group_partial2(r * z, r * r, rbuf(), lt);
        B.sync();
        const float2 t = group_read2(rbuf());
        vz = vbuf(0);
        ++ph;
        ++it;
        conv = t.y <= target;
        beta = __fdividef(t.x, gamma);
        gamma = t.x;
      }
      if (lt == 0) cnt[3] += it;
      if (conv) {
        solved = true;
        xm = x;
      } else {
        flags |= kRowCgFallback;
        if (lt == 0) ++cnt[4];
      }
    }
    if constexpr (!L::kChol) {
      if (!solved) {
        // no tile for this rank: the row goes to the post-pass of the
        // one-CTA-per-row kernel, which writes its result and status
        if (lt == 0) plan.fb_rows[atomicAdd(plan.fb_count, 1)] = (int)u;
        if constexpr (!REG) {
          tc::tc_fence_before();
          tc::mbar_arrive(&c.acc_empty[ab]);
        }
        continue;
      }
    }
    if (lt == 0) ++cnt[0];
    if constexpr (L::kChol) {
      if (!solved) {
        // the system into the tile for the register-tile Cholesky
        B.sync();  // the tile, dg, bv and xv are free; the last reduction has been read
        float *Sr = S + (m < FP ? m : 0) * LDS;
        sys.store(Sr, live);  // every thread (warp-collective TMEM loads); live rows store
        if (m < FP) {
          if (live)
            for (int cc = f; cc < FP; ++cc) Sr[cc] = 0.f;  // padding (and the b_u column)
          bv[m] = bm;
        }
        __syncwarp();
        if (m < FP && !live)
          for (int cc = 0; cc < FP; ++cc) S[m * LDS + cc] = cc == m ? 1.f : 0.f;  // identity block
        B.sync();
        const int res = ws_cholesky<FP>(S, dg, bv, xv, tmp, rd, red + 32, bad, f, reg, a.refine_tol, B);
        if (res == 1) {
          flags |= kRowNotSPD;
          if (lt == 0) ++cnt[2];
        } else if (res == 2) {
          flags |= kRowRefinedF64;
          if (lt == 0) ++cnt[1];
        }
        if (live) xm = xv[m];
        B.sync();
      }
    }
    if constexpr (!REG) {
      // the accumulator may be overwritten now
      tc::tc_fence_before();
      tc::mbar_arrive(&c.acc_empty[ab]);
    }
    if (live) {
      a.dst[u * a.ld_dst + m] = xm;
      if (a.dst_lp) reinterpret_cast<LP *>(a.dst_lp)[u * a.ld_dst_lp + m] = LP(xm);
    }
    if (a.row_flags && lt == 0) a.row_flags[u] = flags;
  }
  if (a.counters && lt == 0) {
    atomicAdd(&a.counters->rows, cnt[0]);
    if (cnt[1]) atomicAdd(&a.counters->refined, cnt[1]);
    if (cnt[2]) atomicAdd(&a.counters->not_spd, cnt[2]);
    if (cnt[3]) atomicAdd(&a.counters->cg_steps, cnt[3]);
    if (cnt[4]) atomicAdd(&a.counters->cg_fallback, cnt[4]);
    if (cnt[5]) atomicAdd(&a.counters->r0_micro, cnt[5]);
  }
}

template <int FP, int NP, typename LP, int NG>
__global__ void __launch_bounds__(ws::threads<NG>(), 1)
rows_tc_ws_kernel(RowsArgs a, uint32_t idesc, TcSolve sv, WsGeom g, WsPlan plan_arg) {
  using L = WsLayout<FP, NP, NG>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned char *base = smem_raw + ((1024 - (tc::smem_u32(smem_raw) & 1023)) & 1023);
  unsigned char *ctrl = base + L::oCtrl;
  WsCtrl c;
  c.full = reinterpret_cast<uint64_t *>(ctrl);
  c.empty = c.full + ws::NS;
  c.acc_full = c.empty + ws::NS;
  c.acc_empty = c.acc_full + ws::kMaxAcc;
  c.row_full = c.acc_empty + ws::kMaxAcc;
  c.row_empty = c.row_full + ws::kRowSlots;
  c.drain = c.row_empty + ws::kRowSlots;
  c.stage_info = reinterpret_cast<uint32_t *>(ctrl + L::kBars);
  c.row_info = reinterpret_cast<int4 *>(ctrl + L::kBars) + ws::NS;
  c.misc = reinterpret_cast<volatile int *>(c.row_info + ws::kRowSlots);
  const int tid = threadIdx.x, warp = tid >> 5;
  const WsPlan &plan = plan_arg;  // stays in the parameter space

  if (tid == 0) {
    for (int i = 0; i < ws::NS; ++i) {
      tc::mbar_init(&c.full[i], ws::kFullCount);
      tc::mbar_init(&c.empty[i], 1);
    }
    for (int b = 0; b < ws::kMaxAcc; ++b) {
      tc::mbar_init(&c.acc_full[b], 1);
      tc::mbar_init(&c.acc_empty[b], 128);
    }
    for (int b = 0; b < ws::kRowSlots; ++b) {
      tc::mbar_init(&c.row_full[b], 1);
      tc::mbar_init(&c.row_empty[b], 128);  // every thread of the taking group
    }
    tc::mbar_init(c.drain, 1);
    c.misc[1] = 0;
    c.misc[3] = 0;  // rows claimed by the solver warpgroups
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == ws::mma_warp<NG>()) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     tc::smem_u32((const void *)&c.misc[0])),
                 "r"(ws::kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  for (int q = tid; q < ws::NS * ws::Dims<FP>::kStageBytes / 16; q += ws::threads<NG>())
    reinterpret_cast<uint4 *>(base)[q] = make_uint4(0, 0, 0, 0);
  tc::fence_proxy_async();
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = (uint32_t)c.misc[0];
  unsigned long long n_empty = 0;

  if (warp == ws::mma_warp<NG>()) {
    if ((tid & 31) == 0) ws_mma<FP>(a, c, base, tmem, idesc, sv.withhold_first && blockIdx.x == 0);
    __syncwarp();
  } else if (warp == ws::prod_warp<NG>() || warp >= ws::prod_warp<NG>() + 2) {
    const int k = warp == ws::prod_warp<NG>() ? 0 : warp - ws::prod_warp<NG>() - 1;
    ws_produce<FP, LP, NG>(a, plan, g, c, base,
                           base + L::oRing + (size_t)k * ws::Dims<FP>::kDI * ws::Dims<FP>::kRingSlot,
                           k, n_empty);
    if ((tid & 31) == 0 && a.counters && n_empty) atomicAdd(&a.counters->rows, n_empty);
  } else if (warp < 4 * NG) {
    unsigned char *mem = base + L::oSolver + (size_t)(warp >> 2) * L::kSolver;
    // Ranks up to 112: the system stays in its TMEM accumulator. Above: the
    // wide solver, rows in registers with one solver warpgroup (255 registers
    // a thread hold a row without spilling), in TMEM otherwise.
    if constexpr (!ws::Dims<FP>::kWide) ws_solve<FP, NP, LP, NG>(a, plan, sv, c, mem, tmem, warp >> 2);
    else ws_solve_wide<FP, NP, LP, NG, NG == 1>(a, plan, sv, c, mem, tmem, warp >> 2);
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == ws::mma_warp<NG>()) {
    tc::tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(ws::kTmemCols));
  }
}

bool tc_ws_supported(int f) { return f >= 16 && f <= 128; }
bool tc_ws_takes(int f, int solver, int jacobi) {
  return tc_ws_supported(f) && (f <= 112 || (solver == 1 && !jacobi));
}

// Load the kernel instance for (f, lp_kind, groups) and set its shared-memory
// attribute without launching it, so that its first real launch (for example
// one the autotuner times) carries no loading cost.
cudaError_t prepare_rows_tc_ws(int f, int lp_kind, int groups) {
  RowsArgs a{};
  a.f = f;
  a.ld_src = tc_padded_ld(f);
  a.src = reinterpret_cast<const void *>(uintptr_t(256));  // never dereferenced
  TcSolve sv{};
  sv.solver = 1;  // every instance takes CG (wide ones only CG)
  sv.groups = groups;
  sv.prepare = 1;
  WsPlan plan;
  plan.nitems = 1;
  plan.part_ld = 132;
  return launch_rows_tc_ws(a, lp_kind, sv, plan, 1, 0);
}
int tc_ws_np(int f) { return ((f + 15) / 16) * 16; }

template <int FP, int NP, typename LP, int NG>
static cudaError_t launch_ws(const RowsArgs &a, int lp_kind, const TcSolve &sv,
                             const WsPlan &plan, int num_sms, cudaStream_t st) {
  using L = WsLayout<FP, NP, NG>;
  static_assert(L::kTotal <= 232448, "227 KB of shared memory per CTA");
  WsGeom g;
  g.nj = a.ld_src / 8;
  constexpr int kMaxLd = ws::Dims<FP>::kWide ? 136 : 120;  // c_r = ld within the stage's atoms
  if (a.ld_src % 8 != 0 || a.ld_src > kMaxLd || NP < a.f || FP < a.f || plan.part_ld < NP + 1)
    return cudaErrorInvalidValue;
  if (ws::Dims<FP>::kWide && (sv.solver != 1 || sv.jacobi)) return cudaErrorNotSupported;
  if ((reinterpret_cast<uintptr_t>(a.src) & 15) != 0) return cudaErrorInvalidValue;
  auto kern = rows_tc_ws_kernel<FP, NP, LP, NG>;
  cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L::kTotal);
  if (err != cudaSuccess || sv.prepare) return err;
  (void)num_sms;
  const int grid = plan.ctas;  // the items were dealt to exactly this many CTAs
  if (grid < 1 || !plan.chol) return cudaErrorInvalidValue;
  const int nmma = ((std::max(NP, a.ld_src + 1) + 15) / 16) * 16;  // B columns incl. c_r
  const uint32_t idesc = tc::make_idesc(lp_kind == kLpBf16 ? 1 : 0, nmma);
  kern<<<(unsigned)grid, ws::threads<NG>(), L::kTotal, st>>>(a, idesc, sv, g, plan);
  return cudaGetLastError();
}

template <int FP, int NP>
static cudaError_t launch_ws_np(const RowsArgs &a, int lp_kind, const TcSolve &sv,
                                const WsPlan &plan, int num_sms, cudaStream_t st) {
  if (sv.groups == 1)
    return lp_kind == kLpBf16 ? launch_ws<FP, NP, __nv_bfloat16, 1>(a, lp_kind, sv, plan, num_sms, st)
                              : launch_ws<FP, NP, __half, 1>(a, lp_kind, sv, plan, num_sms, st);
  if (sv.groups == 3)
    return lp_kind == kLpBf16 ? launch_ws<FP, NP, __nv_bfloat16, 3>(a, lp_kind, sv, plan, num_sms, st)
                              : launch_ws<FP, NP, __half, 3>(a, lp_kind, sv, plan, num_sms, st);
  return lp_kind == kLpBf16 ? launch_ws<FP, NP, __nv_bfloat16, 2>(a, lp_kind, sv, plan, num_sms, st)
                            : launch_ws<FP, NP, __half, 2>(a, lp_kind, sv, plan, num_sms, st);
}

// f in [16, 112]: NP = roundup16(f) accumulator columns are read back per row,
// FP >= f is the Cholesky tile extent.
cudaError_t launch_rows_tc_ws(const RowsArgs &a, int lp_kind, const TcSolve &sv,
                              const WsPlan &plan, int num_sms, cudaStream_t st) {
  const int f = a.f;
  if (!tc_ws_supported(f)) return cudaErrorNotSupported;
  if (plan.nitems <= 0) return cudaSuccess;
  switch (tc_ws_np(f)) {
    case 16: return launch_ws_np<32, 16>(a, lp_kind, sv, plan, num_sms, st);
    case 32: return launch_ws_np<32, 32>(a, lp_kind, sv, plan, num_sms, st);
    case 48: return launch_ws_np<64, 48>(a, lp_kind, sv, plan, num_sms, st);
    case 64: return launch_ws_np<64, 64>(a, lp_kind, sv, plan, num_sms, st);
    case 80: return launch_ws_np<104, 80>(a, lp_kind, sv, plan, num_sms, st);
    case 96: return launch_ws_np<104, 96>(a, lp_kind, sv, plan, num_sms, st);
    case 112: return f <= 104 ? launch_ws_np<104, 112>(a, lp_kind, sv, plan, num_sms, st)
                              : launch_ws_np<112, 112>(a, lp_kind, sv, plan, num_sms, st);
    case 128: return launch_ws_np<128, 128>(a, lp_kind, sv, plan, num_sms, st);
    default: return cudaErrorNotSupported;
  }
}

// ---------------------------------------------------------------------------
// device planning of the work list
// ---------------------------------------------------------------------------
// The work list of a side is built on the device from its row pointers, with
// no copy to the host and no synchronisation:
//   plan_count_kernel  per row: its item count (1, or the chunks of a row
//                      longer than `split`), a histogram of item sizes over
//                      kPlanBins size bins (largest first), and for each split
//                      row its chunk count and first partial slot;
//   plan_scan_kernel   exclusive scan of the histogram (the first rank of each
//                      bin) and the item total;
//   plan_place_kernel  each item's rank (its bin's next free rank: a block
//                      reserves its bin counts in one atomic per bin, then
//                      ranks its rows in shared memory) and its place: ranks
//                      are dealt to the CTAs in rounds of alternating
//                      direction, and within the CTA the order zigzags
//                      between its largest and smallest items, so rows that load
//                      the producers (many ratings) alternate with rows that
//                      load the solvers (few ratings).
// Items of one size bin are ranked in no fixed order; every row is solved the
// same way wherever it is placed (the partial sums of a split row are added in
// chunk order), so the results do not depend on the order.
namespace {
constexpr int kPlanBins = 4096;
constexpr int kPlanThreads = 512;

struct PlanHdr {
  unsigned long long extra;  // items beyond one per row (extra chunks of split rows)
  int nheavy, nslots, nitems, pad;
};

struct PlanDev {
  const int64_t *ptr;
  int64_t begin, count;
  int grid, hmax, smax;
  int64_t imax;  // capacity of items
  int *error;  // optional: bit 2 set when the row pointers break the bounds below
  PlanHdr *hdr;
  unsigned *hist, *cursor;
  int *heavy_row, *heavy_nchunks, *heavy_base;
  unsigned *heavy_count;
  WorkItem *items;
};

__device__ __forceinline__ int64_t plan_split(const PlanDev &p) {
  const int64_t nnz = p.ptr[p.begin + p.count] - p.ptr[p.begin];
  const int64_t q = (int64_t)kPlanSplitDiv * p.grid;
  const int64_t s = (nnz + q - 1) / q;
  return s > 8192 ? s : 8192;
}
static_assert(kPlanBins == 4 * 1024, "plan_scan_kernel: 1024 threads of four bins");

// A row's rating count; a decreasing row pointer (a malformed CSR) counts as
// an empty row rather than a negative size.
__device__ __forceinline__ int64_t plan_deg(const PlanDev &p, int64_t r) {
  const int64_t d = p.ptr[p.begin + r + 1] - p.ptr[p.begin + r];
  return d > 0 ? d : 0;
}
// Size bins, largest first: items shorter than kPlanExact ratings (most rows
// of power-law matrices) get a bin of their own size, so they are ordered
// exactly; longer ones share kPlanBins - kPlanExact bins spread linearly up to
// `split`.
constexpr int kPlanExact = 3072;
__device__ __forceinline__ int plan_bin(int64_t size, int64_t split) {
  if (size < kPlanExact) return kPlanBins - 1 - (int)size;
  constexpr int kCoarse = kPlanBins - kPlanExact;
  const int64_t span = split - kPlanExact + 1;  // split >= 8192 > kPlanExact
  return (int)((split - size) * kCoarse / span);
}
__device__ __forceinline__ void plan_rows_of_block(const PlanDev &p, int64_t &r0, int64_t &r1) {
  const int64_t per = (p.count + gridDim.x - 1) / gridDim.x;
  r0 = (int64_t)blockIdx.x * per;
  r1 = r0 + per < p.count ? r0 + per : p.count;
}

__global__ void __launch_bounds__(kPlanThreads) plan_count_kernel(PlanDev p) {
  __shared__ unsigned hs[kPlanBins];
  for (int b = threadIdx.x; b < kPlanBins; b += blockDim.x) hs[b] = 0;
  __syncthreads();
  const int64_t split = plan_split(p);
  int64_t r0, r1;
  plan_rows_of_block(p, r0, r1);
  for (int64_t r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
    const int64_t d = plan_deg(p, r);
    if (d > split) {
      const int64_t nch = (d + split - 1) / split;
      atomicAdd(&hs[0], (unsigned)(nch - 1));  // full chunks
      atomicAdd(&hs[plan_bin(d - (nch - 1) * split, split)], 1u);
      const int h = atomicAdd(&p.hdr->nheavy, 1);
      const int hb = atomicAdd(&p.hdr->nslots, (int)nch);
      if (h >= p.hmax || hb + nch > p.smax) {  // only a malformed CSR gets here
        p.hdr->pad = 1;
        continue;
      }
      p.heavy_row[h] = (int)r;
      p.heavy_nchunks[h] = (int)nch;
      p.heavy_base[h] = hb;
      p.heavy_count[h] = 0;
      atomicAdd(&p.hdr->extra, (unsigned long long)(nch - 1));
    } else {
      atomicAdd(&hs[plan_bin(d, split)], 1u);
    }
  }
  __syncthreads();
  for (int b = threadIdx.x; b < kPlanBins; b += blockDim.x)
    if (hs[b]) atomicAdd(&p.hist[b], hs[b]);
}

// One block of 1024 threads: each scans four consecutive bins.
__global__ void __launch_bounds__(1024) plan_scan_kernel(PlanDev p) {
  __shared__ unsigned part[1024];
  const int t = threadIdx.x;
  unsigned v[4], s = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    v[k] = p.hist[4 * t + k];
    s += v[k];
  }
  part[t] = s;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {
    const unsigned add = t >= o ? part[t - o] : 0u;
    __syncthreads();
    part[t] += add;
    __syncthreads();
  }
  unsigned run = part[t] - s;  // exclusive prefix of this thread's four bins
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    p.cursor[4 * t + k] = run;
    run += v[k];
  }
  if (t == 0) {
    // Row pointers that broke the plan's bounds leave no plan at all
    // (nothing is solved) and raise the error word, rather than a partial one.
    const int64_t n = p.count + (int64_t)p.hdr->extra;
    const bool bad = p.hdr->pad != 0 || n > p.imax;
    p.hdr->nitems = bad ? 0 : (int)n;
    if (bad && p.error) atomicOr(p.error, 2);
  }
}

// Rank k (largest first) goes to round q = k / G of the deal, and is its
// CTA's q-th largest of nc items. Rounds run across the CTAs in alternating
// directions (a snake), so no CTA takes the largest item of every round; the
// last round, when partial, runs forward, so that CTA c still holds
// ceil((N - c) / G) items (the kernel reads CTA c's items at c, c + G, ...
// below N). Within the CTA the order zigzags between its largest and smallest
// items (slots 0, 2, 4, ... take the largest, 1, 3, 5, ... the smallest).
__device__ __forceinline__ void plan_put(const PlanDev &p, int64_t k, int64_t N, const WorkItem &w) {
  const int64_t G = p.grid, q = k / G;
  const bool partial = N % G != 0 && q == N / G;
  const int64_t c = ((q & 1) && !partial) ? G - 1 - k % G : k % G, nc = (N - c + G - 1) / G;
  const int64_t j = q < (nc + 1) / 2 ? 2 * q : 2 * (nc - 1 - q) + 1;  // zigzag slot
  p.items[c + j * G] = w;
}

__global__ void __launch_bounds__(kPlanThreads) plan_place_kernel(PlanDev p) {
  __shared__ unsigned cnt[kPlanBins];
  __shared__ unsigned base[kPlanBins];
  for (int b = threadIdx.x; b < kPlanBins; b += blockDim.x) cnt[b] = 0;
  __syncthreads();
  const int64_t split = plan_split(p), N = p.hdr->nitems;
  if (N == 0) return;  // a rejected plan (block-uniform)
  int64_t r0, r1;
  plan_rows_of_block(p, r0, r1);
  for (int64_t r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
    const int64_t d = plan_deg(p, r);
    if (d <= split) atomicAdd(&cnt[plan_bin(d, split)], 1u);
  }
  __syncthreads();
  for (int b = threadIdx.x; b < kPlanBins; b += blockDim.x) {
    base[b] = cnt[b] ? atomicAdd(&p.cursor[b], cnt[b]) : 0u;
    cnt[b] = 0;
  }
  __syncthreads();
  for (int64_t r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
    const int64_t s = p.ptr[p.begin + r], d = plan_deg(p, r);
    if (d > split) continue;
    const int b = plan_bin(d, split);
    WorkItem w;
    w.s = s;
    w.e = s + d;
    w.u = (int)(p.begin + r);
    w.deg = (int)d;
    w.part = -1;
    w.heavy = -1;
    plan_put(p, (int64_t)base[b] + atomicAdd(&cnt[b], 1u), N, w);
  }
  // the chunks of split rows, a split row per block at a time
  const int nheavy = p.hdr->nheavy;
  for (int h = blockIdx.x; h < nheavy; h += gridDim.x) {
    const int64_t r = p.heavy_row[h], s = p.ptr[p.begin + r], e = s + plan_deg(p, r);
    const int nch = p.heavy_nchunks[h], hb = p.heavy_base[h];
    for (int ch = threadIdx.x; ch < nch; ch += blockDim.x) {
      WorkItem w;
      w.s = s + ch * split;
      w.e = min(e, s + (ch + 1) * split);
      w.u = (int)(p.begin + r);
      w.deg = (int)(e - s);
      w.part = hb + ch;
      w.heavy = h;
      plan_put(p, (int64_t)atomicAdd(&p.cursor[plan_bin(w.e - w.s, split)], 1u), N, w);
    }
  }
}

struct PlanLayout {
  size_t oHdr, oHist, oCur, oHr, oHn, oHb, oHc, oItems, oPart, oChol, oFb, oFbc, total;
  PlanLayout(int64_t count, int grid, int np) {
    auto al = [](size_t x) { return (x + 255) / 256 * 256; };
    // A row of d > split ratings becomes ceil(d / split) < d / split + 1
    // chunks, and split >= nnz / (D grid), D = kPlanSplitDiv: fewer than
    // D grid split rows, fewer than 2 D grid chunks of them, fewer than
    // count + D grid items.
    const size_t D = kPlanSplitDiv;
    const size_t hmax = D * (size_t)grid + 1, smax = 2 * D * (size_t)grid,
                 imax = (size_t)count + D * (size_t)grid;
    size_t o = 0;
    oHdr = o; o += al(sizeof(PlanHdr));
    oHist = o; o += al(4 * kPlanBins);
    oCur = o; o += al(4 * kPlanBins);
    oHr = o; o += al(4 * hmax);
    oHn = o; o += al(4 * hmax);
    oHb = o; o += al(4 * hmax);
    oHc = o; o += al(4 * hmax);
    oItems = o; o += al(sizeof(WorkItem) * imax);
    oPart = o; o += al(sizeof(float) * smax * 128 * (size_t)(np + 4) + 16);
    oChol = o; o += al(sizeof(float) * (size_t)grid * ws::kMaxGroups * kCholFloats);
    oFb = o; o += al(4 * (size_t)count);  // rows deferred to the post-pass (ranks above 112)
    oFbc = o; o += al(8);
    total = o;
  }
};

int plan_grid(int64_t count, int grid) {
  return (int)std::max<int64_t>(1, std::min<int64_t>(grid, count));
}
}  // namespace

size_t plan_ws_bytes(int64_t count, int grid, int np) {
  return PlanLayout(count, plan_grid(count, grid), np).total;
}

cudaError_t plan_ws(const int64_t *d_row_ptr, int64_t begin, int64_t count, int grid, int np,
                    int src_rows, void *mem, size_t mem_bytes, WsPlan *plan, int *error,
                    cudaStream_t st) {
  *plan = WsPlan();
  plan->src_rows = src_rows;
  plan->part_ld = np + 4;
  if (count <= 0) return cudaSuccess;
  if (count > INT32_MAX) return cudaErrorInvalidValue;
  // Every CTA of the launch gets at least one item: there are at least as
  // many items as rows.
  grid = plan_grid(count, grid);
  const PlanLayout L(count, grid, np);
  if (!mem || mem_bytes < L.total || (reinterpret_cast<uintptr_t>(mem) & 255) != 0)
    return cudaErrorInvalidValue;
  char *d = static_cast<char *>(mem);
  PlanDev p;
  p.ptr = d_row_ptr;
  p.begin = begin;
  p.count = count;
  p.grid = grid;
  p.hmax = kPlanSplitDiv * grid + 1;
  p.smax = 2 * kPlanSplitDiv * grid;
  p.imax = count + (int64_t)kPlanSplitDiv * grid;
  p.error = error;
  p.hdr = reinterpret_cast<PlanHdr *>(d + L.oHdr);
  p.hist = reinterpret_cast<unsigned *>(d + L.oHist);
  p.cursor = reinterpret_cast<unsigned *>(d + L.oCur);
  p.heavy_row = reinterpret_cast<int *>(d + L.oHr);
  p.heavy_nchunks = reinterpret_cast<int *>(d + L.oHn);
  p.heavy_base = reinterpret_cast<int *>(d + L.oHb);
  p.heavy_count = reinterpret_cast<unsigned *>(d + L.oHc);
  p.items = reinterpret_cast<WorkItem *>(d + L.oItems);
  cudaError_t e = cudaMemsetAsync(d, 0, L.oCur, st);  // header and histogram
  if (e != cudaSuccess) return e;
  const int sms = device_sm_count();
  const unsigned blocks = (unsigned)std::max<int64_t>(
      1, std::min<int64_t>(2LL * (sms > 0 ? sms : 148), (count + kPlanThreads - 1) / kPlanThreads));
  plan_count_kernel<<<blocks, kPlanThreads, 0, st>>>(p);
  plan_scan_kernel<<<1, 1024, 0, st>>>(p);
  plan_place_kernel<<<blocks, kPlanThreads, 0, st>>>(p);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  plan->items = p.items;
  plan->nitems = (int)std::min<int64_t>(INT32_MAX, count + 4LL * grid);  // upper bound
  plan->nitems_dev = &p.hdr->nitems;
  plan->heavy_nchunks = p.heavy_nchunks;
  plan->heavy_base = p.heavy_base;
  plan->heavy_count = p.heavy_count;
  plan->partial = reinterpret_cast<float *>(d + L.oPart);
  plan->chol = reinterpret_cast<float *>(d + L.oChol);
  plan->ctas = grid;
  plan->fb_rows = reinterpret_cast<int *>(d + L.oFb);
  plan->fb_count = reinterpret_cast<int *>(d + L.oFbc);
  plan->rows = count;
  return cudaSuccess;
}

}  // namespace als
