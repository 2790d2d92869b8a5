// Mixed-precision latent sampler whose row Grams run on the tcgen05 tensor cores (KP = 32).
// k_gram_tc<true> (the sampler of a BPMF / Macau mode) accumulates every sampled row's Gram
// V^T V and right-hand side on the tensor cores and finishes the row in its epilogue (Lambda +
// alpha G, FP32 Cholesky, solves, noise), so a row's Gram never leaves the SM.  k_gram_tc<false>
// stores the Grams to HBM as records instead, for finishes that run as a separate kernel: the
// univariate prior (k_finish_one_tc), the batched problems (batch.cu), and k_finish_tc.
//
// k_gram_tc.  Four sampler rows ("a group") share each MMA.  For a k-block of 16 entries per
// row, the producers gather the four rows' BF16 other-factor vectors (64 B each, by CSR column
// index) with 16-byte cp.async copies into one shared-memory stage of five SW64 MN-major column
// blocks (32 elements wide, two K-atoms of 8 k-rows x 64 B): block p holds row p's 32 latent
// values, block 4 holds the rows' weights w = (y - mean) * alpha split into two BF16 parts, the
// rounded weight in elements 0..3 and the remainder w - bf16(w) in elements 4..7.  One
// tcgen05.mma (M = 128, N = 160, K = 16, BF16 in, FP32 accumulate in TMEM) per stage adds
//     D[32p + i][32q + j] += sum_k X_p[k][i] X_q[k][j],   D[32p + i][128 + q] += sum_k X_p[k][i] w_q[k]
// whose diagonal blocks p == q are the four rows' Grams and whose columns 128 + p and 132 + p
// sum to row p's right-hand side sum v (y - mean) alpha (the off-diagonal blocks are not used);
// the weights thus enter with 16 significant bits, not BF16's 8.  D row r lives
// in TMEM lane r, so the warp of quadrant p reads row p's Gram with one 32x32b load.
// (A TMA tile::gather4 variant of the producers was measured slower: a gather4 of 64-byte rows
// into a 64B-swizzled stage must start on the 512-byte swizzle period, which leaves half of each
// K-atom empty and doubles the MMAs, and each warp issues one TMA instruction per ~70-90 cycles.)
//
// The CSR stream is the padded packed array of the mode: each row's (column, weight) entries
// start on a 16-entry boundary and are padded to a multiple of 16 with (N_other, 0) sentinels;
// a sentinel gathers the zero row N_other of the BF16 factor, and so does a row slot with no
// entries left in a k-block.
//
// Warp roles (one persistent CTA per SM: 20 warps in the fused kernel, 16 in the records kernel):
//   warps 0-7   producers: the k-blocks go through the pipeline in blocks of kBlk = 4 (global
//               k-blocks 4b .. 4b + 3 in the stages of block b % 6), with one barrier handshake
//               per block, not per k-block: a barrier wait or arrive costs tens to ~150 cycles,
//               as much as the work of a k-block.  Warp w fills column block r = w % 4 of the
//               stages of the blocks b = w / 4 (mod 2): per block it takes row r's 4 x 16 CSR
//               entries from the CSR ring of its parity, issues two 16-byte cp.async per lane
//               and k-block (lane l: chunk l % 4 of entries l / 4 and l / 4 + 8) as one commit
//               group and stores the weights; one block later it waits for that group, fences
//               the async proxy and arrives on the block's "full" barrier (4 arrivals).
//   warp 8      MMA: allocates TMEM (512 columns: three accumulators of 160 columns); lane 0
//               alone waits for each block, issues its MMAs, releases the block's stages
//               (tcgen05.commit -> "empty") and publishes finished accumulators (tcgen05.commit
//               -> "acc full").  One wait per block, not per MMA: on B200 an mbarrier wait (or
//               any shared-memory read) issued right after a tcgen05.mma took ~150 cycles,
//               about as long as the M=128, N=160, K=16 MMA, which left the tensor core idle
//               half the time when every k-block had its own wait.
//   warp 9      scheduler: takes 4 tasks per group from the work queue (four claims in flight)
//               and publishes the group descriptors into a ring of kDesc slots, so that the
//               queue atomics and task loads stay off the MMA warp; it claims a new group only
//               while fewer than kAheadKb k-blocks of its published groups wait for the MMAs.
//   warps 10-11 CSR loaders, one per block parity: walk the group descriptors and, up to kCsr
//               blocks of their parity ahead, copy the four 128-byte row segments of each of the
//               block's k-blocks with one 16-byte cp.async per lane into the ring, with a meta
//               record (block index, valid row slots per k-block, end) for the producers.
//   warps 12-15 epilogue / drainers (warp w reads TMEM quadrant w % 4 = row slot): TMEM ->
//               registers, release the accumulator and the group's descriptor slot ("desc
//               free"); a part of a split row goes to the part's scratch slot as an FP64
//               partial.  Records kernel: the row's FP32 Gram and rhs go to its Gram record.
//               Fused kernel: the quadrant is staged in shared memory, in a ring of four groups
//               per quadrant, for the finisher of the same quadrant.
//   warps 16-19 finishers (fused kernel only, warpgroup 4, which takes registers from the other
//               four by setmaxnreg): finisher qd takes four staged groups at a time, hands the
//               ring slots back once the rows are in registers, and finishes the four rows
//               together (quarter q of the warp: the row of group 4i + q; the quad routines of
//               warp_finish.cuh), so the factors of one batch overlap the MMAs and the staging
//               of the next groups.  A row whose FP32 factor fails is redone by the whole warp
//               in FP64 from the row's CSR entries and BF16 latents (retry_row_from_csr), with
//               the warp's work area in global memory (SampleParams::retry_work).
// Every barrier wait is bounded by a clock budget (SampleParams::wait_cycles, about 2 s by
// default); on expiry the CTA raises an abort flag, all roles leave their loops, the MMA lane
// drains its MMAs (a wait of the full default budget), TMEM is freed and the status word reports
// a timeout.
//
// k_finish_tc.  One warp per four rows: the Gram records (or the FP64 sums of split rows' parts,
// in part order, written by k_sum_parts), then the FP32 quad Cholesky and solves of
// warp_finish.cuh with an FP64 retry of the same Gram.  After the fused kernel it finishes the
// split rows only, from a compact list of their records.
#include <cuda_bf16.h>

#include "common.cuh"
#include "kernels.h"
#include "rng.cuh"
#include "warp_finish.cuh"

namespace mg {
namespace {

constexpr int kRowSlots = 4;
constexpr int kParity = 2;                          // producers per row slot
constexpr int kProducers = kRowSlots * kParity;     // warps 0-7 (warpgroups 0 and 1)
constexpr int kMmaWarp = kProducers;                // warp 8   (warpgroup 2)
constexpr int kSchedWarp = kProducers + 1;          // warp 9
constexpr int kCsrWarp0 = kProducers + 2;           // warps 10-11
constexpr int kEpiWarp0 = kProducers + 4;           // warps 12-15 (warpgroup 3)
constexpr int kFinWarp0 = kProducers + 8;           // warps 16-19 (warpgroup 4, fused kernel)
constexpr int kTcThreads = (kProducers + 8) * 32;   // records kernel: 16 warps
constexpr int kTcThreadsFused = kTcThreads + 128;   // fused kernel: 20 warps
// Fused kernel: registers per thread after the warpgroups rebalance (setmaxnreg) from the 96 of
// the launch (65,536 / 640 rounded down to a multiple of 8): warpgroups 0-3 give theirs up to the
// finishers, whose four-row finish keeps 80 matrix entries per lane plus the dependency chains
// of four matrices in flight.  The split must fit the launch allocation:
// 16 warps x 32 x 56 + 4 x 32 x 256 = 61,440 <= 640 x 96.
constexpr int kLaunchRegs = 96;
constexpr int kOtherRegs = 56;
constexpr int kFinRegs = 256;
static_assert((kTcThreadsFused - 128) * kOtherRegs + 128 * kFinRegs <=
                  kTcThreadsFused * kLaunchRegs,
              "register split exceeds the launch allocation");
static_assert(kEpiWarp0 % 4 == 0 && kTcThreads - kEpiWarp0 * 32 == 128 &&
                  kFinWarp0 * 32 == kTcThreads,
              "the epilogue, then the finishers, must be the last warpgroups");
constexpr int kStages = 24;               // gather stages in flight (even: stage s has parity s % 2)
// Stages are handed from the producers to the MMA lane in blocks of kBlk consecutive k-blocks,
// one "full" and one "empty" barrier per block: a barrier wait issued right after a tcgen05.mma
// takes about as long as the MMA itself, so the MMA lane waits once per kBlk MMAs.
constexpr int kBlk = 4;
constexpr int kBlocks = kStages / kBlk;
constexpr int kBlockBytes = 2 * 512;      // one column block: 2 K-atoms x 512 B
constexpr int kStageBytes = 5 * kBlockBytes;
constexpr int kSlots = 3;                 // TMEM accumulators
constexpr int kSlotCols = 160;            // columns of one accumulator (N = 160)
constexpr int kCsr = 4;                   // CSR ring slots per parity (blocks of that parity ahead)
constexpr int kDesc = 64;                 // group descriptor ring
// The scheduler claims a new group from the work queue only while fewer than kAheadKb k-blocks
// of its published groups still wait for the MMAs: the queue then hands out groups as each CTA
// consumes them, which balances the CTAs' work (a 64-group ring claimed at once fixed most of
// the assignment at the start and left CTAs' end times 20-30% apart).  It must exceed the
// k-blocks the producers and loaders run ahead of the MMAs.
constexpr int kAheadKb = 96;
constexpr long long kWaitCycles = 4000000000LL;  // ~2 s at 2 GHz
constexpr int kGramRec = 32 * 32 + 32;    // Gram record: 32 x 32 row-major Gram, then the rhs
static_assert(kStages % kParity == 0, "a stage's k-blocks all have the same parity");
static_assert(kStages % kBlk == 0, "stages come in whole blocks");

struct GroupDesc {
  int row[4];
  int len[4];
  long long begin[4];
  int part[4];
  int nparts[4];
  int slot[4];
  int nkb;     // k-blocks of the group (>= 1; the stop group has kBlk, which completes the last
               // block the MMA lane waits for)
  int stop;    // 1: no more work
};

// Descriptor ring: the scheduler rewrites slot g % kDesc for group g + kDesc only after the
// epilogue released group g ("desc free"), and the producers, the MMA lane and the epilogue all
// read a group's descriptor before the epilogue releases it.  The ring must cover the groups
// the producers run ahead of the MMAs (at most kStages + kCsr k-blocks) and the accumulators.
static_assert(kDesc > kStages + kParity * kCsr * kBlk + kSlots + 1, "descriptor ring too small");
static_assert(kAheadKb > kStages + kParity * kCsr * kBlk + kBlk, "claim window too small");

constexpr int kMetaEnd = 1 << 16;  // meta flag: no more blocks of this parity

struct TcShared {
  uint64_t full[kBlocks];      // one producer arrival per row slot and k-block of the block
  uint64_t empty[kBlocks];     // tcgen05.commit after the block's MMAs
  uint64_t acc_full[kSlots];
  uint64_t acc_empty[kSlots];  // 4 epilogue warps
  uint64_t drain;
  uint64_t never;              // nothing arrives here (SampleParams::wait_test)
  uint64_t desc_full[kDesc];   // scheduler -> producers, MMA, epilogue
  uint64_t desc_free[kDesc];   // epilogue (4 warps) -> scheduler
  uint64_t csr_full[kParity][kCsr];   // 32 cp.async completions + the loader's meta arrive
  uint64_t csr_empty[kParity][kCsr];  // the 4 producers of the parity are done with the slot
  int2 meta[kParity][kCsr];           // {block index, valid bits (bit 4u + r) | kMetaEnd}
  alignas(16) uint2 csr[kParity][kCsr][kBlk][4][16];  // CSR entries of one block: [kb][slot][16]
  uint32_t tmem_base;
  int abort;
  int mma_kb;             // k-blocks the MMA lane has taken (written after each block)
  long long wait_cycles;  // budget of one barrier wait (SampleParams::wait_cycles, or kWaitCycles)
  GroupDesc desc[kDesc];
};

__device__ __forceinline__ uint32_t su32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(b)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(su32(b)) : "memory");
}

__device__ __forceinline__ bool mbar_test(uint64_t* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred P1;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, P1;\n\t}"
      : "=r"(ok)
      : "r"(su32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Like mbar_test, but a thread whose phase is not complete may be suspended by the hardware
// for up to `ns` nanoseconds while it waits, instead of returning at once (no issue slots are
// spent while suspended).
__device__ __forceinline__ bool mbar_test_suspend(uint64_t* b, uint32_t parity, uint32_t ns) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred P1;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2, %3;\n\t"
      "selp.b32 %0, 1, 0, P1;\n\t}"
      : "=r"(ok)
      : "r"(su32(b)), "r"(parity), "r"(ns)
      : "memory");
  return ok != 0;
}

// Slow path of mbar_wait: suspended tries of up to 20 us, the abort flag and the clock budget
// checked between them.  Inlined like every device function of the fused kernel: a call from
// warpgroups that run with different register counts (setmaxnreg) does not allocate.
__device__ __forceinline__ bool mbar_wait_slow(uint64_t* b, uint32_t parity, TcShared* sh, Ctl* ctl) {
  const long long t0 = clock64();
  const long long budget = sh->wait_cycles;
  for (;;) {
    if (mbar_test_suspend(b, parity, 20000u)) return true;
    if (*(volatile int*)&sh->abort) return false;
    if (clock64() - t0 > budget) {
      atomicOr(&ctl->status, kStatTimeout);
      *(volatile int*)&sh->abort = 1;
      return false;
    }
  }
}

// Bounded wait on phase `parity`: false on timeout or when another role aborted.
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity, TcShared* sh, Ctl* ctl) {
  if (mbar_test(b, parity)) return true;
  return mbar_wait_slow(b, parity, sh, ctl);
}

// Bounded wait until the MMA lane has taken `target` k-blocks (polled with sleeps; false on
// timeout or abort, like mbar_wait).
__device__ __forceinline__ bool wait_mma_kb(TcShared* sh, int target, Ctl* ctl) {
  if (*(volatile int*)&sh->mma_kb >= target) return true;
  const long long t0 = clock64();
  const long long budget = sh->wait_cycles;
  for (;;) {
    __nanosleep(256);
    if (*(volatile int*)&sh->mma_kb >= target) return true;
    if (*(volatile int*)&sh->abort) return false;
    if (clock64() - t0 > budget) {
      atomicOr(&ctl->status, kStatTimeout);
      *(volatile int*)&sh->abort = 1;
      return false;
    }
  }
}

// Waits for every cp.async of this thread.
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
// 16-byte asynchronous copy global -> shared (L2 only).
__device__ __forceinline__ void cp16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(su32(dst)), "l"(src) : "memory");
}
// Arrive on `b` once every earlier cp.async of this thread has completed (the barrier's count
// includes this arrival).
__device__ __forceinline__ void cp_arrive_noinc(uint64_t* b) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(su32(b)) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait_group() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// SW64 MN-major shared-memory matrix descriptor: MN-atom stride 2048 B (LBO), K-atom stride
// 512 B (SBO), descriptor version 1, layout type 4 (64-byte swizzle).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)(kBlockBytes >> 4) << 16) |
         ((uint64_t)(512 >> 4) << 32) | (1ull << 46) | (4ull << 61);
}

// kind::f16 instruction descriptor: D FP32, A/B BF16, A/B MN-major, N = 160, M = 128.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) |
                            ((160u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t acc) {
  const uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
      ::"r"(d_tmem), "l"(a), "l"(b), "r"(kIdesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* b) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   su32(b))
               : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, "
      "%29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
        "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
        "=r"(r[31])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ float tmem_ld1(uint32_t taddr) {
  uint32_t r;
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%1];" : "=r"(r) : "r"(taddr));
  return __uint_as_float(r);
}

__device__ __forceinline__ void tmem_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Byte offset of element (mn, j) of a stage, j = entry 0..15 of the row's k-block (bf16
// elements; SW64 MN-major: 64 B per k-row, entry j in K-atom j / 8, k-row j % 8, 16-byte chunk
// index XOR (k-row / 2) % 4).
__device__ __forceinline__ uint32_t stage_off(int mn, int j) {
  const int a = mn >> 5, e = mn & 31, c = e >> 3, b = j >> 3, r = j & 7;
  return (uint32_t)(a * kBlockBytes + b * 512 + r * 64 + ((c ^ ((r >> 1) & 3)) << 4) +
                    ((e & 7) << 1));
}

// Writes the descriptor of group g (tasks t0 .. t0 + 3; lanes 0-3 hold their task in `tk`,
// valid when `has`) and publishes it; `nkb_out` = its k-blocks.  Returns true for the stop group
// (t0 past the end).
__device__ __forceinline__ bool publish_group(TcShared* sh, int g, int t0, int ntasks,
                                              const RowTask& tk, bool has, int lane,
                                              int& nkb_out) {
  GroupDesc& d = sh->desc[g % kDesc];
  const bool stop = t0 >= ntasks;
  int rkb = 0;
  if (lane < 4) {
    d.row[lane] = has ? tk.row : -1;
    d.len[lane] = has ? tk.len : 0;
    d.begin[lane] = has ? tk.begin : 0;
    d.part[lane] = has ? tk.part : 0;
    d.nparts[lane] = has ? tk.nparts : 1;
    d.slot[lane] = has ? tk.slot : 0;
    rkb = has ? tk.len >> 4 : 0;  // the k-blocks of each row (its padded length / 16)
  }
  int nkb = rkb;
#pragma unroll
  for (int o = 1; o < 4; o <<= 1) nkb = max(nkb, __shfl_xor_sync(0xffffffffu, nkb, o));
  nkb = __shfl_sync(0xffffffffu, nkb, 0);
  nkb_out = stop ? kBlk : max(nkb, 1);
  if (lane == 0) {
    d.nkb = nkb_out;
    d.stop = stop ? 1 : 0;
  }
  __syncwarp();
  if (lane == 0) mbar_arrive(&sh->desc_full[g % kDesc]);
  return stop;
}

// A producer's position in the flattened (group, k-block) sequence, restricted to the k-blocks
// of its parity: group g, k-block kb of it, global k-block index t.
struct Cursor {
  int g, kb, t;
  int nkb, rkb;
  long long beg;
  bool stop, end;
};

// Reads group c.g's descriptor (waiting for it to be published).  False on timeout / abort.
__device__ __forceinline__ bool cursor_load(Cursor& c, TcShared* sh, Ctl* ctl, int r) {
  if (!mbar_wait(&sh->desc_full[c.g % kDesc], (uint32_t)((c.g / kDesc) & 1), sh, ctl)) return false;
  const GroupDesc& d = sh->desc[c.g % kDesc];
  c.nkb = d.nkb;
  c.stop = d.stop != 0;
  c.beg = d.begin[r];
  c.rkb = d.len[r] >> 4;
  return true;
}

// Moves the cursor `step` k-blocks on (crossing group boundaries); c.end once it passes the
// stop group.  False on timeout / abort.
__device__ __forceinline__ bool cursor_advance(Cursor& c, int step, TcShared* sh, Ctl* ctl, int r) {
  c.kb += step;
  c.t += step;
  while (c.kb >= c.nkb) {
    if (c.stop) {
      c.end = true;
      return true;
    }
    c.kb -= c.nkb;
    c.g++;
    if (!cursor_load(c, sh, ctl, r)) return false;
  }
  return true;
}

// ---------------------------------------------------------------------------------------------
// Row finish shared by the fused epilogue and k_finish_tc.
constexpr int kFinWarps = 8;
constexpr int kLc = 36;                 // L^T leading dimension
constexpr int kFinWork = 32 * 36 * 8;   // per warp: the FP64 retry's L^T (leading dimension kLc)

// Entry (c, j) of MM = Lambda + alpha G in FP32 from (float) Lambda(c, j) and G(c, j); the
// identity beyond K.
__device__ __forceinline__ float mm_entry(float lam, float g, float alpha_f, int c, int j, int K) {
  return (c < K && j < K) ? lam + alpha_f * g : (c == j ? 1.f : 0.f);
}

// Per-launch constants of the row finish in shared memory: Lambda in FP64 (row stride 33) and
// FP32 (row stride kLc), and Lambda mu in FP64.
struct FinConst {
  double Lam[32 * 33];
  double lmu[32];
  alignas(16) float LamF[32 * kLc];
};

// Fills FinConst with `nthreads` threads (thread index t), `bar` ordering the two steps.
template <typename Bar>
__device__ __forceinline__ void fin_const_fill(FinConst* fc, const SampleParams& p, int t,
                                               int nthreads, Bar bar) {
  const int K = p.K;
  for (int e = t; e < 32 * 32; e += nthreads) {
    const int i = e / 32, j = e % 32;
    const double v = (i < K && j < K) ? p.Lambda[i + j * K] : 0.0;
    fc->Lam[i * 33 + j] = v;
    fc->LamF[i * kLc + j] = (float)v;
  }
  bar();
  if (t < 32) {
    double s = 0.0;
    if (t < K)
      for (int j = 0; j < K; j++) s += fc->Lam[t * 33 + j] * p.mu[j];
    fc->lmu[t] = s;
  }
  bar();
}

// Rows i, i + 8, i + 16, i + 24 of the quarter's MM = Lambda + alpha G (FP32, the quad layout of
// warp_finish.cuh) from its Gram rows at gp (row-major, 32 floats a row; staged: each row's
// 16-byte chunk c stored at chunk c ^ (row % 8), which keeps the quarter's reads and the
// epilogue's writes free of bank conflicts), d0[k] = the diagonal entry of row i + 8k.
template <bool kStaged>
__device__ __forceinline__ void quad_load_mm(const FinConst* fc, const float* gp, int i, int K,
                                             float alpha_f, float (&a)[80], float (&d0)[4]) {
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const int r = i + 8 * k;
    d0[k] = 1.f;
#pragma unroll
    for (int c4 = 0; c4 < 2 * (k + 1); c4++) {
      const float* src = gp + r * 32 + 4 * (kStaged ? (c4 ^ i) : c4);
      const float4 g = kStaged ? *reinterpret_cast<const float4*>(src)
                               : __ldcg(reinterpret_cast<const float4*>(src));
      const float4 m = *reinterpret_cast<const float4*>(fc->LamF + r * kLc + 4 * c4);
      const float gv[4] = {g.x, g.y, g.z, g.w}, mv[4] = {m.x, m.y, m.z, m.w};
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const int c = 4 * c4 + u;
        const float v = mm_entry(mv[u], gv[u], alpha_f, r, c, K);
        a[qoff(k) + c] = v;
        if (c == r) d0[k] = v;
      }
    }
  }
}

// Right-hand sides of components i + 8k of `row` in FP32: the Gram rhs (rhs[c]) + Lambda mu
// (Macau: Lambda (mu + Uhat[row])), summed in FP64.
template <bool kStaged>
__device__ __forceinline__ void quad_rhs(const SampleParams& p, const FinConst* fc,
                                         const float* rhs, int row, int i, float (&b)[4]) {
  const int K = p.K;
  double m[4] = {0.0, 0.0, 0.0, 0.0};
  if (p.uhat) {
    for (int j = 0; j < K; j++) {
      const double mj = p.mu[j] + p.uhat[(size_t)row * 32 + j];
#pragma unroll
      for (int k = 0; k < 4; k++)
        if (i + 8 * k < K) m[k] += fc->Lam[(i + 8 * k) * 33 + j] * mj;
    }
  } else {
#pragma unroll
    for (int k = 0; k < 4; k++) m[k] = fc->lmu[i + 8 * k];
  }
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const float rv = kStaged ? rhs[i + 8 * k] : __ldcg(rhs + i + 8 * k);
    double rl = (double)rv;
    rl += m[k];
    b[k] = (float)rl;
  }
}

// Finishes four rows, one per quarter (the quarter's row `row`, < 0: takes no part, computing on
// row rw's draws): MM from its Gram at gp, FP32 factor, solves and the draw, the latents stored
// when the factor held.  `loaded()` runs once the Grams are in registers.  Returns the ballot of lanes whose quarter has a row and a failed factor
// (bit 8q for quarter q).
template <bool kStaged, typename Loaded>
__device__ __forceinline__ unsigned quad_finish(const SampleParams& p, const FinConst* fc,
                                                const float* gp, int row, int rw, float alpha_f,
                                                uint32_t sweep, int lane, Loaded loaded) {
  const int i = lane & 7;
  const int K = p.K;
  float a[80], d0[4], rinv[4] = {1.f, 1.f, 1.f, 1.f}, b[4], z[4];
  quad_load_mm<kStaged>(fc, gp, i, K, alpha_f, a, d0);
  quad_rhs<kStaged>(p, fc, gp + 32 * 32, rw, i, b);
  loaded();  // the Grams at gp are no longer read
  quad_noise(p, rw, K, i, sweep, z);
  const bool ok = quad_factor(a, rinv, i, d0);
  quad_solve(a, rinv, b, z, i);
  if (ok && row >= 0) {
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const int c = i + 8 * k;
      if (c < K) {
        p.out_f32[(size_t)row * 32 + c] = b[k];
        p.out_bf16[(size_t)row * 32 + c] = __float2bfloat16_rn(b[k]);
      }
    }
  }
  return __ballot_sync(0xffffffffu, !ok && row >= 0);
}

// FP64 redo of one row whose FP32 factor failed, by the whole warp (lane = component), from the
// same FP32 Gram record (the two-kernel path): rhs + Lambda mu recomputed in FP64, then
// warp_finish_f64.
__device__ __noinline__ void retry_row_from_record(const SampleParams& p, const FinConst* fc,
                                                   const float* rec, int row, uint32_t sweep,
                                                   unsigned char* work) {
  const int lane = threadIdx.x & 31;
  const int K = p.K;
  double rl = 0.0;
  if (lane < K) {
    rl = (double)__ldcg(rec + 32 * 32 + lane);
    double m = 0.0;
    if (p.uhat) {
      for (int j = 0; j < K; j++) m += fc->Lam[lane * 33 + j] * (p.mu[j] + p.uhat[(size_t)row * 32 + j]);
    } else {
      m = fc->lmu[lane];
    }
    rl += m;
  }
  if (lane == 0) atomicAdd(&p.ctl->retries[p.mode], 1u);
  const bool ok = warp_finish_f64<32, float>(rec, 32, fc->Lam, rl, p, row, sweep, work);
  if (!ok && lane == 0) {
    atomicOr(&p.ctl->status, kStatCholFail);
    atomicCAS(&p.ctl->bad_row, -1, row);
  }
  __syncwarp();
}

// FP64 redo of one row whose FP32 factor failed, by the whole warp (lane = component): the
// Gram sum v v^T and rhs sum v w re-accumulated in FP64 from the row's padded CSR entries
// [begin, begin + len) and the BF16 latents they gather (the inputs of the tensor-core Gram,
// without its FP32 rounding), then MM = Lambda + alpha G, the FP64 warp Cholesky and solves with
// the row's keyed draws.  Counts a retry; a failed FP64 factor raises kStatCholFail.
__device__ __forceinline__ void retry_row_from_csr(const SampleParams& p, const FinConst* fc,
                                                int row, long long begin, int len,
                                                uint32_t sweep, unsigned char* work) {
  const int lane = threadIdx.x & 31;
  const int K = p.K;
  const __nv_bfloat16* V = reinterpret_cast<const __nv_bfloat16*>(p.other);
  const float wscale = (float)packed_scale(p);
  double g[32];
#pragma unroll
  for (int j = 0; j < 32; j++) g[j] = 0.0;
  double b = 0.0;
  for (int e = 0; e < len; e++) {
    const uint2 ent = p.packed[begin + e];
    const float vi = __bfloat162float(V[(size_t)ent.x * 32 + lane]);
    const double w = (double)(__uint_as_float(ent.y) * wscale);
    b = fma((double)vi, w, b);
#pragma unroll
    for (int j = 0; j < 32; j++) g[j] = fma((double)vi, (double)__shfl_sync(0xffffffffu, vi, j), g[j]);
  }
  const double alpha = noise_alpha(p);
  double a[32], d0 = 1.0, rinv = 1.0;
#pragma unroll
  for (int j = 0; j < 32; j++) {
    a[j] = (lane < K && j < K) ? fc->Lam[lane * 33 + j] + alpha * g[j] : (lane == j ? 1.0 : 0.0);
    if (j == lane) d0 = a[j];
  }
  double rr = 0.0;
  if (lane < K) {
    rr = b;
    if (p.uhat) {
      for (int j = 0; j < K; j++)
        rr += fc->Lam[lane * 33 + j] * (p.mu[j] + p.uhat[(size_t)row * 32 + j]);
    } else {
      rr += fc->lmu[lane];
    }
  }
  const double z = row_noise(p, row, K, lane, sweep);
  if (lane == 0) atomicAdd(&p.ctl->retries[p.mode], 1u);
  double* Lc = reinterpret_cast<double*>(work);
  __syncwarp();
  if (!warp_factor<double, 32>(a, rinv, lane, 0.0, d0, Lc, kLc)) {
    if (lane == 0) {
      atomicOr(&p.ctl->status, kStatCholFail);
      atomicCAS(&p.ctl->bad_row, -1, row);
    }
    return;
  }
  const double x = warp_solve<double, 32>(a, rinv, rr, lane, Lc, kLc, z);
  if (lane < K) {
    p.out_f32[(size_t)row * 32 + lane] = (float)x;
    p.out_bf16[(size_t)row * 32 + lane] = __float2bfloat16_rn((float)x);
  }
  __syncwarp();
}

// What the fused epilogue needs of its quadrant's task in a group.
struct EpiTask {
  long long begin;
  int row, len, part, nparts, pslot, stop;
};

// Fused epilogue: waits for group g's accumulator, reads this warp's quadrant qd (lane l: Gram
// row l of the group's row slot qd and the rhs component l) and the slot's task, then releases
// the accumulator and the descriptor.  False on timeout / abort.
__device__ __forceinline__ bool epi_take(TcShared* sh, Ctl* ctl, uint32_t tmem, int g, int qd,
                                         int lane, EpiTask& t, float (&gr)[32], float& rhs) {
  const int slot = g % kSlots;
  if (!mbar_wait(&sh->acc_full[slot], (uint32_t)((g / kSlots) & 1), sh, ctl)) return false;
  if (!mbar_wait(&sh->desc_full[g % kDesc], (uint32_t)((g / kDesc) & 1), sh, ctl)) return false;
  tc_fence_after();
  const GroupDesc& d = sh->desc[g % kDesc];
  t.stop = d.stop;
  t.row = d.row[qd];
  t.len = d.len[qd];
  t.begin = d.begin[qd];
  t.part = d.part[qd];
  t.nparts = d.nparts[qd];
  t.pslot = d.slot[qd];
  __syncwarp();
  if (lane == 0) mbar_arrive(&sh->desc_free[g % kDesc]);
  rhs = 0.f;
  if (!t.stop) {
    const uint32_t lanes = (uint32_t)(32 * qd) << 16;
    tmem_ld32(tmem + lanes + (uint32_t)(slot * kSlotCols + 32 * qd), gr);
    const float rhs_hi = tmem_ld1(tmem + lanes + (uint32_t)(slot * kSlotCols + 128 + qd));
    const float rhs_lo = tmem_ld1(tmem + lanes + (uint32_t)(slot * kSlotCols + 132 + qd));
    tmem_wait_ld();
    rhs = rhs_hi + rhs_lo;
  } else {
#pragma unroll
    for (int j = 0; j < 32; j++) gr[j] = 0.f;
  }
  tc_fence_before();
  __syncwarp();
  if (lane == 0) mbar_arrive(&sh->acc_empty[slot]);
  return true;
}

// A split row's part: its FP32 partial Gram (lane = Gram row) and rhs to the part's FP64 scratch
// slot, summed in part order by k_sum_parts.
__device__ __forceinline__ void store_part(const SampleParams& p, const EpiTask& t,
                                           const float (&gr)[32], float rhs, int lane) {
  double* sp = p.scratch + (size_t)(t.pslot + t.part) * kGramRec;
#pragma unroll
  for (int j = 0; j < 32; j++) sp[lane * 32 + j] = (double)gr[j];
  sp[32 * 32 + lane] = (double)rhs;
}

// Staging of one group's quadrant for the quad finish: the 32 Gram rows (row r's 16-byte chunk c
// at chunk c ^ (r % 8)), then the 32 rhs values.
constexpr int kStageRec = 32 * 32 + 32;

__device__ __forceinline__ void stage_rows(float* st, const float (&gr)[32], float rhs, int lane) {
#pragma unroll
  for (int c4 = 0; c4 < 8; c4++)
    *reinterpret_cast<float4*>(st + lane * 32 + 4 * (c4 ^ (lane & 7))) =
        make_float4(gr[4 * c4], gr[4 * c4 + 1], gr[4 * c4 + 2], gr[4 * c4 + 3]);
  st[32 * 32 + lane] = rhs;
}

// Shared memory of the fused kernel beyond TcShared: the finish constants and, per TMEM
// quadrant qd, a ring of four staged Grams (slot q: group 4i + q) with their tasks, handed from
// drainer qd to finisher qd by a pair of barriers per slot.
struct FusedShared {
  FinConst fc;
  alignas(16) float stage[4][4 * kStageRec];
  long long begin[4][4];
  int row[4][4], len[4][4], stop[4][4];
  uint64_t staged[4][4];  // drainer qd staged slot q (1 arrival)
  uint64_t sfree[4][4];   // finisher qd has read slot q (1 arrival)
};

template <bool kFused>
__global__ void __launch_bounds__(kFused ? kTcThreadsFused : kTcThreads, 1)
    k_gram_tc(const SampleParams p, float* gram) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // layout: stages (1024-aligned) | TcShared | FusedShared (fused kernel)
  unsigned char* stages = smem_raw;
  TcShared* sh = reinterpret_cast<TcShared*>(stages + (size_t)kStages * kStageBytes);
  FusedShared* fs = reinterpret_cast<FusedShared*>(reinterpret_cast<unsigned char*>(sh) +
                                                   (sizeof(TcShared) + 15) / 16 * 16);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // The stage descriptors' 64-byte swizzle pattern assumes 1024-byte aligned stages.
  if ((su32(stages) & 1023u) != 0) {
    if (threadIdx.x == 0) atomicOr(&p.ctl->status, kStatTimeout);
    return;
  }

  // ---- set-up ----
  // zero the stages once: weight elements 8..31 stay zero
  for (int e = threadIdx.x; e < kStages * kStageBytes / 16; e += blockDim.x)
    reinterpret_cast<uint4*>(stages)[e] = make_uint4(0u, 0u, 0u, 0u);
  if (threadIdx.x == 0) {
    for (int b = 0; b < kBlocks; b++) {
      mbar_init(&sh->full[b], kRowSlots);  // one arrive per producer (the block's copies landed)
      mbar_init(&sh->empty[b], 1);
    }
    for (int s = 0; s < kSlots; s++) {
      mbar_init(&sh->acc_full[s], 1);
      mbar_init(&sh->acc_empty[s], 4);
    }
    mbar_init(&sh->drain, 1);
    mbar_init(&sh->never, 1);
    for (int d = 0; d < kDesc; d++) {
      mbar_init(&sh->desc_full[d], 1);
      mbar_init(&sh->desc_free[d], 4);
    }
    for (int h = 0; h < kParity; h++)
      for (int c = 0; c < kCsr; c++) {
        mbar_init(&sh->csr_full[h][c], 33);
        mbar_init(&sh->csr_empty[h][c], kRowSlots);
      }
    sh->abort = 0;
    sh->mma_kb = 0;
    if constexpr (kFused) {
      for (int qd = 0; qd < 4; qd++)
        for (int q = 0; q < 4; q++) {
          mbar_init(&fs->staged[qd][q], 1);
          mbar_init(&fs->sfree[qd][q], 1);
        }
    }
    sh->wait_cycles = p.wait_cycles > 0 ? p.wait_cycles : kWaitCycles;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == kMmaWarp) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     su32(&sh->tmem_base)),
                 "r"(512));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  fence_proxy_async();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = sh->tmem_base;

  // Fused kernel: each role branch starts with its warpgroup's register rebalance (setmaxnreg
  // is executed by all warps of a warpgroup at the same instruction, so warpgroup 2's three
  // roles share one branch).
  if (warp < kProducers) {
    if constexpr (kFused) asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(kOtherRegs));
    // ================= producer of row slot r, parity h =================
    // Blocks b = h (mod 2): per block the producer takes row r's 4 x 16 CSR entries from the
    // CSR ring of its parity and, for each k-block u of the block, issues two 16-byte cp.async
    // per lane (lane l: chunk l % 4 of entries l / 4 and l / 4 + 8) and stores the 16 weights;
    // the block's copies form one cp.async group.  One block later it waits for that group,
    // fences the async proxy (its copies and weights before the tensor cores read them) and
    // arrives on the block's "full" barrier.
    const int r = warp % kRowSlots, h = warp / kRowSlots;
    const int ch = lane & 3, e0 = lane >> 2;
    // this lane's weight element in a stage: lanes 0-15 hold the BF16 weight of entry lane % 16
    // in B column 128 + r, lanes 16-31 the BF16 remainder w - bf16(w) in column 132 + r, so the
    // two accumulated right-hand-side columns add up to sum v w with w kept to 16 mantissa bits
    const uint32_t woff = stage_off(128 + r + 4 * (lane >> 4), lane & 15);
    const uint32_t o0 = stage_off(32 * r + 8 * ch, e0), o1 = stage_off(32 * r + 8 * ch, e0 + 8);
    const __nv_bfloat16* V = reinterpret_cast<const __nv_bfloat16*>(p.other);
    const unsigned sentinel = (unsigned)p.nother;  // the zero row of the BF16 factor
    const float wscale = (float)packed_scale(p);     // 1 unless the noise is adaptive
    int pend = -1;  // block whose "full" arrive is pending
    for (int i = 0;; i++) {
      const int slot = i % kCsr;
      if (!mbar_wait(&sh->csr_full[h][slot], (uint32_t)((i / kCsr) & 1), sh, p.ctl)) break;
      const int2 m = sh->meta[h][slot];
      if (m.y & kMetaEnd) break;
      unsigned col0[kBlk], col1[kBlk];
      __nv_bfloat16 w_st[kBlk];
#pragma unroll
      for (int u = 0; u < kBlk; u++) {
        const bool v = (m.y >> (4 * u + r)) & 1;
        const uint2* e = sh->csr[h][slot][u][r];
        col0[u] = v ? e[e0].x : sentinel;
        col1[u] = v ? e[e0 + 8].x : sentinel;
        const float w = v ? __uint_as_float(e[lane & 15].y) * wscale : 0.f;
        const __nv_bfloat16 w_hi = __float2bfloat16_rn(w);
        w_st[u] = lane < 16 ? w_hi : __float2bfloat16_rn(w - __bfloat162float(w_hi));
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&sh->csr_empty[h][slot]);  // the entries are in registers
      const int blk = m.x % kBlocks;
      if (!mbar_wait(&sh->empty[blk], (uint32_t)(((m.x / kBlocks) & 1) ^ 1), sh, p.ctl)) break;
#pragma unroll
      for (int u = 0; u < kBlk; u++) {
        unsigned char* sbase = stages + (size_t)(blk * kBlk + u) * kStageBytes;
        cp16(sbase + o0, V + (size_t)col0[u] * 32 + 8 * ch);
        cp16(sbase + o1, V + (size_t)col1[u] * 32 + 8 * ch);
        *reinterpret_cast<__nv_bfloat16*>(sbase + woff) = w_st[u];
      }
      cp_commit();
      if (pend >= 0) {
        // the previous block's copies have landed (this block's group may remain)
        cp_wait_group<1>();
        fence_proxy_async();
        __syncwarp();
        if (lane == 0) mbar_arrive(&sh->full[pend]);
      }
      pend = blk;
    }
    // the pending block
    cp_wait_all();
    fence_proxy_async();
    __syncwarp();
    if (pend >= 0 && lane == 0) mbar_arrive(&sh->full[pend]);
  } else if (warp < kEpiWarp0) {
    if constexpr (kFused) asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(kOtherRegs));
    if (warp == kMmaWarp) {
    // ================= MMA issuer (lane 0) =================
    if (lane == 0) {
      // test hook: a wait that runs out (the abort path then ends every role)
      bool ok = !p.wait_test || mbar_wait(&sh->never, 0, sh, p.ctl);
      // the open group: g, its accumulator slot, k-blocks done / of the group, stop flag
      int g = 0, kb = 0, nkb = 0, slot = 0, stop = 0;
      uint32_t d_tmem = tmem;
      // opens group g: waits for its accumulator to be free and its descriptor published
      auto open_group = [&]() -> bool {
        slot = g % kSlots;
        if (g >= kSlots &&
            !mbar_wait(&sh->acc_empty[slot], (uint32_t)(((g / kSlots) & 1) ^ 1), sh, p.ctl))
          return false;
        if (!mbar_wait(&sh->desc_full[g % kDesc], (uint32_t)((g / kDesc) & 1), sh, p.ctl))
          return false;
        tc_fence_after();
        const GroupDesc& d = sh->desc[g % kDesc];
        nkb = d.nkb;
        stop = d.stop;
        kb = 0;
        d_tmem = tmem + (uint32_t)(slot * kSlotCols);
        // the stop group has no MMAs: its accumulator is published at once (the epilogue
        // reads only the descriptor's stop flag)
        if (stop) mma_commit(&sh->acc_full[slot]);
        return true;
      };
      ok = ok && open_group();
      for (int b = 0; ok && !stop; b++) {
        const int blk = b % kBlocks;
        if (!mbar_wait(&sh->full[blk], (uint32_t)((b / kBlocks) & 1), sh, p.ctl)) break;
        tc_fence_after();
        // unrolled, each MMA with its own descriptor registers (measured on B200: the rolled
        // loop kept the MMA lane busy ~1,200 cycles per block of four, this one ~800)
        const uint32_t s0 = su32(stages + (size_t)blk * kBlk * kStageBytes);
        if (kb + kBlk <= nkb) {
          // the whole block belongs to the open group: four MMAs in a row with no branch
          // between them (on long rows about 13% faster than the general loop below)
#pragma unroll
          for (int u = 0; u < kBlk; u++) {
            const uint64_t dsc = smem_desc(s0 + (uint32_t)(u * kStageBytes));
            mma_bf16(d_tmem, dsc, dsc, (kb + u) > 0 ? 1u : 0u);
          }
          kb += kBlk;
          if (kb == nkb) {
            mma_commit(&sh->acc_full[slot]);
            g++;
            if (!open_group()) ok = false;
          }
        } else
#pragma unroll
        for (int u = 0; u < kBlk; u++) {
          if (ok && !stop) {
            const uint64_t dsc = smem_desc(s0 + (uint32_t)(u * kStageBytes));
            mma_bf16(d_tmem, dsc, dsc, kb > 0 ? 1u : 0u);
            if (++kb == nkb) {
              mma_commit(&sh->acc_full[slot]);
              g++;
              if (!open_group()) ok = false;
            }
          }
        }
        mma_commit(&sh->empty[blk]);
        *(volatile int*)&sh->mma_kb = (b + 1) * kBlk;
      }
      // drain: wait for every issued MMA before TMEM is released
      mma_commit(&sh->drain);
      const long long t0 = clock64();
      while (!mbar_test(&sh->drain, 0) && clock64() - t0 < kWaitCycles) __nanosleep(128);
    }
    __syncwarp();
    } else if (warp == kSchedWarp) {
    // ================= scheduler =================
    // lane 0 keeps four queue claims in flight (q[0] oldest); the next group's tasks are
    // loaded while the current group is published
    int q[4] = {0, 0, 0, 0};
    if (lane == 0) {
#pragma unroll
      for (int j = 0; j < 4; j++) q[j] = (int)atomicAdd(&p.ctl->queue[p.qslot], 4u);
    }
    int t_cur = __shfl_sync(0xffffffffu, q[0], 0);
    RowTask tk_cur = p.tasks[min(t_cur + lane, p.ntasks - 1)];
    int pub_kb = 0;  // k-blocks of the published groups
    for (int g = 0;; g++) {
      if (g >= kDesc && !mbar_wait(&sh->desc_free[g % kDesc],
                                   (uint32_t)(((g / kDesc) - 1) & 1), sh, p.ctl))
        break;
      if (!wait_mma_kb(sh, pub_kb - kAheadKb, p.ctl)) break;
      if (lane == 0) {
        q[0] = q[1];
        q[1] = q[2];
        q[2] = q[3];
        if (t_cur < p.ntasks) q[3] = (int)atomicAdd(&p.ctl->queue[p.qslot], 4u);
      }
      const int t_nxt = __shfl_sync(0xffffffffu, q[0], 0);
      const RowTask tk_nxt = p.tasks[min(t_nxt + lane, p.ntasks - 1)];
      const bool has = lane < 4 && t_cur + lane < p.ntasks;
      int nkb = 0;
      if (publish_group(sh, g, t_cur, p.ntasks, tk_cur, has, lane, nkb)) break;
      pub_kb += nkb;
      t_cur = t_nxt;
      tk_cur = tk_nxt;
    }
    } else {
    // ================= CSR loader of parity h =================
    // Blocks b = h (mod 2), up to kCsr of them ahead: for each k-block u of the block, lane l
    // copies entries 2 (l % 8) .. + 1 of row slot l / 8 (one 16-byte cp.async) into the ring;
    // the meta record carries the block index and the valid (row slot, k-block) bits.  The
    // cursor then skips the other parity's block.
    const int h = warp - kCsrWarp0, rs = lane >> 3, c2 = 2 * (lane & 7);
    Cursor c{0, 0, 0, 0, 0, 0, false, false};
    bool ok = cursor_load(c, sh, p.ctl, rs) && cursor_advance(c, h * kBlk, sh, p.ctl, rs);
    for (int i = 0; ok; i++) {
      const int slot = i % kCsr;
      if (i >= kCsr &&
          !mbar_wait(&sh->csr_empty[h][slot], (uint32_t)(((i / kCsr) - 1) & 1), sh, p.ctl))
        break;
      const bool end = c.end;  // the block starts past the stop group: nothing more to do
      int flags = 0;
#pragma unroll
      for (int u = 0; u < kBlk; u++) {
        const bool v = !c.end && !c.stop && c.kb < c.rkb;
        if (v) cp16(&sh->csr[h][slot][u][rs][c2], p.packed + c.beg + 16LL * c.kb + c2);
        const unsigned vm = __ballot_sync(0xffffffffu, v);
#pragma unroll
        for (int q = 0; q < 4; q++) flags |= (int)((vm >> (8 * q)) & 1u) << (4 * u + q);
        if (ok) ok = cursor_advance(c, 1, sh, p.ctl, rs);
      }
      cp_arrive_noinc(&sh->csr_full[h][slot]);
      if (lane == 0) sh->meta[h][slot] = make_int2(h + kParity * i, end ? kMetaEnd : flags);
      __syncwarp();
      if (lane == 0) mbar_arrive(&sh->csr_full[h][slot]);
      if (end) break;
      if (ok) ok = cursor_advance(c, (kParity - 1) * kBlk, sh, p.ctl, rs);
    }
    cp_wait_all();
    }
  } else if (warp < kFinWarp0) {
    const int qd = warp & 3;  // TMEM quadrant = row slot of the group
    if constexpr (kFused) {
      asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(kOtherRegs));
      // ================= drainer of quadrant qd: accumulators -> staging ring =================
      // group g goes to ring slot q = g % 4 of the quadrant once finisher qd has read the
      // slot's previous group; the accumulator and the descriptor are released as soon as they
      // are read, so the MMAs of the next groups overlap the finish of the staged ones.
      for (int g = 0;; g++) {
        const int q = g & 3;
        if (g >= 4 &&
            !mbar_wait(&fs->sfree[qd][q], (uint32_t)(((g >> 2) - 1) & 1), sh, p.ctl))
          break;
        EpiTask t;
        float gr[32], rhs;
        if (!epi_take(sh, p.ctl, tmem, g, qd, lane, t, gr, rhs)) break;
        if (!t.stop) {
          stage_rows(fs->stage[qd] + q * kStageRec, gr, rhs, lane);
          if (t.row >= 0 && t.nparts > 1) store_part(p, t, gr, rhs, lane);
        }
        if (lane == 0) {
          fs->row[qd][q] = (!t.stop && t.row >= 0 && t.nparts == 1) ? t.row : -1;
          fs->begin[qd][q] = t.begin;
          fs->len[qd][q] = t.len;
          fs->stop[qd][q] = t.stop;
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&fs->staged[qd][q]);
        if (t.stop) break;
      }
    } else {
      // ================= epilogue: accumulators -> Gram records =================
      for (int g = 0;; g++) {
        const int slot = g % kSlots;
        if (!mbar_wait(&sh->acc_full[slot], (uint32_t)((g / kSlots) & 1), sh, p.ctl)) break;
        if (!mbar_wait(&sh->desc_full[g % kDesc], (uint32_t)((g / kDesc) & 1), sh, p.ctl)) break;
        tc_fence_after();
        const GroupDesc& d = sh->desc[g % kDesc];
        const int stop = d.stop;
        const int row = d.row[qd];
        const int part = d.part[qd], nparts = d.nparts[qd], pslot = d.slot[qd];
        __syncwarp();
        if (lane == 0) mbar_arrive(&sh->desc_free[g % kDesc]);
        float gr[32];
        float rhs = 0.f;
        if (!stop) {
          const uint32_t lanes = (uint32_t)(32 * qd) << 16;
          tmem_ld32(tmem + lanes + (uint32_t)(slot * kSlotCols + 32 * qd), gr);
          const float rhs_hi = tmem_ld1(tmem + lanes + (uint32_t)(slot * kSlotCols + 128 + qd));
          const float rhs_lo = tmem_ld1(tmem + lanes + (uint32_t)(slot * kSlotCols + 132 + qd));
          tmem_wait_ld();
          rhs = rhs_hi + rhs_lo;
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&sh->acc_empty[slot]);
        if (stop) break;
        if (row < 0) continue;
        if (nparts > 1) {
          double* sp = p.scratch + (size_t)(pslot + part) * kGramRec;
#pragma unroll
          for (int j = 0; j < 32; j++) sp[lane * 32 + j] = (double)gr[j];
          sp[32 * 32 + lane] = (double)rhs;
        } else {
          float* gp = gram + (size_t)row * kGramRec;
          const int w = p.row_width ? p.row_width[row] : 32;  // rows and columns the finish reads
          if (lane < w) {
#pragma unroll
            for (int j = 0; j < 32; j += 4)
              if (j < w)
                *reinterpret_cast<float4*>(gp + lane * 32 + j) =
                    make_float4(gr[j], gr[j + 1], gr[j + 2], gr[j + 3]);
            gp[32 * 32 + lane] = rhs;
          }
        }
      }
    }
  } else {
    if constexpr (kFused) {
      asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" ::"n"(kFinRegs));
      // ================= finisher of quadrant qd: staged Grams -> finished rows =================
      // four groups at a time (ring slots 0-3 of the quadrant), quarter q the row of group
      // 4i + q; the slots go back to the drainer once the rows are in registers.  A row whose
      // FP32 factor fails is redone in FP64 from its CSR entries, with this warp's work area in
      // global memory (the ring may already hold the next groups).
      const int qd = warp - kFinWarp0;
      fin_const_fill(&fs->fc, p, threadIdx.x - kFinWarp0 * 32, 128,
                     [] { asm volatile("bar.sync 1, 128;" ::: "memory"); });
      const float alpha_f = (float)noise_alpha(p);
      const uint32_t sweep = p.ctl->sweep;
      float* stage = fs->stage[qd];
      unsigned char* work = reinterpret_cast<unsigned char*>(
          p.retry_work + (size_t)(blockIdx.x * 4 + qd) * (kFinWork / sizeof(double)));
      bool done = false;
      for (int b = 0; !done; b++) {
        int nq = 0;
        for (int q = 0; q < 4; q++) {
          if (!mbar_wait(&fs->staged[qd][q], (uint32_t)(b & 1), sh, p.ctl)) {
            done = true;
            nq = 0;  // aborted: nothing is finished
            break;
          }
          if (fs->stop[qd][q]) {
            done = true;
            break;
          }
          nq = q + 1;
        }
        int rrow[4];
        long long rbeg[4];
        int rlen[4];
        int first = -1;
#pragma unroll
        for (int q = 0; q < 4; q++) {
          rrow[q] = q < nq ? fs->row[qd][q] : -1;
          rbeg[q] = fs->begin[qd][q];
          rlen[q] = fs->len[qd][q];
          if (first < 0 && rrow[q] >= 0) first = rrow[q];
        }
        const auto release = [&] {
          __syncwarp();
          if (lane == 0)
            for (int q = 0; q < nq; q++) mbar_arrive(&fs->sfree[qd][q]);
        };
        if (first < 0) {  // nothing to finish (done ends the loop)
          release();
          continue;
        }
        const int qq = lane >> 3;
        const int row = rrow[qq & 3];
        const unsigned fails = quad_finish<true>(p, &fs->fc, stage + qq * kStageRec, row,
                                                 row >= 0 ? row : first, alpha_f, sweep, lane,
                                                 release);
        __syncwarp();
#pragma unroll
        for (int q = 0; q < 4; q++)
          if ((fails >> (8 * q)) & 1u)
            retry_row_from_csr(p, &fs->fc, rrow[q], rbeg[q], rlen[q], sweep, work);
        __syncwarp();
      }
    }
  }
  // ---- tear-down ----
  tc_fence_before();
  __syncthreads();
  if (warp == kMmaWarp) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
  }
}

// ---------------------------------------------------------------------------------------------
// k_sum_parts: one warp per split row: its parts' FP64 partial Grams summed in part order, one
// entry at a time, and rounded once into an FP32 Gram record (lane i: Gram row i): the row's own
// record, or with `compact` record w of a list of the split rows' records.
__global__ void __launch_bounds__(256)
    k_sum_parts(const double* __restrict__ scratch, const int4* __restrict__ split_rows,
                int nsplit, float* __restrict__ gram, int compact) {
  const int lane = threadIdx.x & 31;
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= nsplit) return;
  const int4 sr = split_rows[w];  // {row, parts, scratch slot of part 0, unused}
  const double* s0 = scratch + (size_t)sr.z * kGramRec;
  float* gp = gram + (size_t)(compact ? w : sr.x) * kGramRec;
  for (int j = 0; j < 32; j++) {
    double acc = 0.0;
    for (int prt = 0; prt < sr.y; prt++) acc += __ldcg(s0 + (size_t)prt * kGramRec + lane * 32 + j);
    gp[lane * 32 + j] = (float)acc;
  }
  double rs = 0.0;
  for (int prt = 0; prt < sr.y; prt++) rs += __ldcg(s0 + (size_t)prt * kGramRec + 32 * 32 + lane);
  gp[32 * 32 + lane] = (float)rs;
}

// k_finish_tc: one warp per four rows (rows 4w .. 4w + 3 for w = warp, warp + total warps, ...),
// quarter q finishing row 4w + q with the quad routines from the row's Gram record.  Rows are
// 0 .. nrows - 1 with record r, or with a list the rows list[i].x with record i (the split rows
// after the fused kernel).  A row whose FP32 factorisation fails is redone in FP64 by the whole
// warp from the same record.
__global__ void __launch_bounds__(kFinWarps * 32, 2)
    k_finish_tc(const SampleParams p, const float* __restrict__ gram,
                const int4* __restrict__ list, int nlist) {
  extern __shared__ __align__(16) unsigned char fsm[];
  FinConst* fc = reinterpret_cast<FinConst*>(fsm);
  unsigned char* works = fsm + (sizeof(FinConst) + 15) / 16 * 16;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t sweep = p.ctl->sweep;
  fin_const_fill(fc, p, threadIdx.x, blockDim.x, [] { __syncthreads(); });
  const float alpha_f = (float)noise_alpha(p);
  unsigned char* work = works + (size_t)warp * kFinWork;
  const int n = list ? nlist : p.nrows;
  const int stride = gridDim.x * kFinWarps;
  for (int w = blockIdx.x * kFinWarps + warp; 4 * w < n; w += stride) {
    const int idx = 4 * w + (lane >> 3);
    const bool have = idx < n;  // the last quarters of a short final group only follow along
    const int iw = have ? idx : 4 * w;
    const int rw = list ? list[iw].x : iw;
    const unsigned fails = quad_finish<false>(p, fc, gram + (size_t)iw * kGramRec, have ? rw : -1,
                                              rw, alpha_f, sweep, lane, [] {});
    __syncwarp();
    for (int q = 0; q < 4; q++)
      if ((fails >> (8 * q)) & 1u) {
        const int fi = 4 * w + q;
        retry_row_from_record(p, fc, gram + (size_t)fi * kGramRec, list ? list[fi].x : fi, sweep,
                              work);
      }
    __syncwarp();
  }
}

// k_finish_one_tc: the univariate prior's finish (one_gs_warp) from the Gram records, one warp
// per row (rows warp, warp + total warps, ...); lane d reads row d of the record.
__global__ void __launch_bounds__(256)
    k_finish_one_tc(const SampleParams p, const float* __restrict__ gram) {
  const int lane = threadIdx.x & 31;
  const uint32_t sweep = p.ctl->sweep;
  const int warps = gridDim.x * (blockDim.x >> 5);
  for (int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); row < p.nrows;
       row += warps) {
    const float* gp = gram + (size_t)row * kGramRec;
    float g[32];
#pragma unroll
    for (int j = 0; j < 32; j += 4) {
      const float4 v = __ldcg(reinterpret_cast<const float4*>(gp + lane * 32 + j));
      g[j] = v.x;
      g[j + 1] = v.y;
      g[j + 2] = v.z;
      g[j + 3] = v.w;
    }
    const double c = (double)__ldcg(gp + 32 * 32 + lane);
    const double u0 = lane < p.K ? (double)p.out_f32[(size_t)row * 32 + lane] : 0.0;
    const double un = one_gs_warp<32, float>(g, c, u0, p, row, sweep, lane);
    if (lane < p.K) {
      p.out_f32[(size_t)row * 32 + lane] = (float)un;
      p.out_bf16[(size_t)row * 32 + lane] = __float2bfloat16_rn((float)un);
    }
  }
}

}  // namespace

size_t tc_retry_work_doubles(int num_sms) {
  return (size_t)num_sms * 4 * (kFinWork / sizeof(double));
}

size_t tc_smem_bytes(bool fused) {
  return (size_t)kStages * kStageBytes + (sizeof(TcShared) + 15) / 16 * 16 +
         (fused ? sizeof(FusedShared) : 0);
}

namespace {
// Opt-in shared memory sizes, set once per device and kernel.
template <typename Kern>
void set_smem(Kern k, size_t bytes, bool (&configured)[64]) {
  int dev = 0;
  MG_CUDA(cudaGetDevice(&dev));
  if (!configured[dev & 63]) {
    MG_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    configured[dev & 63] = true;
  }
}
constexpr size_t kFinSmem = (sizeof(FinConst) + 15) / 16 * 16 + (size_t)kFinWarps * kFinWork;
static_assert((size_t)kStages * kStageBytes + sizeof(TcShared) + 16 + sizeof(FusedShared) <=
                  227 * 1024,
              "fused tensor-core sampler exceeds the shared memory of one CTA");
}  // namespace

bool launch_gram_tc(const SampleParams& p, float* gram, const int4* split_rows, int nsplit,
                    int KP, cudaStream_t s, int num_sms, cudaEvent_t mid) {
  if (KP != 32 || p.packed == nullptr) return false;
  if (p.ntasks == 0) throw MgError(MG_ERR_STATE, "tensor-core Gram kernel without tasks");
  static bool configured[64] = {false};
  const size_t smem = tc_smem_bytes(false);
  set_smem(k_gram_tc<false>, smem, configured);
  k_gram_tc<false><<<num_sms, kTcThreads, smem, s>>>(p, gram);
  MG_CUDA(cudaGetLastError());
  if (mid) MG_CUDA(cudaEventRecord(mid, s));
  if (nsplit > 0) {
    k_sum_parts<<<(nsplit + 7) / 8, 256, 0, s>>>(p.scratch, split_rows, nsplit, gram, 0);
    MG_CUDA(cudaGetLastError());
  }
  return true;
}

bool launch_sample_tc(const SampleParams& p, float* gram, const int4* split_rows, int nsplit,
                      int KP, cudaStream_t s, int num_sms, cudaEvent_t mid, bool fused) {
  if (KP != 32 || p.packed == nullptr) return false;
  if (p.ntasks == 0) {  // an empty row range: nothing to sample
    if (mid) MG_CUDA(cudaEventRecord(mid, s));
    return true;
  }
  static bool configured_fin[64] = {false}, configured_fused[64] = {false};
  set_smem(k_finish_tc, kFinSmem, configured_fin);
  if (fused && !p.one) {
    // the fused kernel finishes every unsplit row; split rows: parts summed into a compact list
    // of records, then finished from there
    const size_t smem = tc_smem_bytes(true);
    set_smem(k_gram_tc<true>, smem, configured_fused);
    // the warpgroups' register rebalance needs the launch allocation it was sized for
    static int launch_regs = 0;
    if (launch_regs == 0) {
      cudaFuncAttributes fa{};
      MG_CUDA(cudaFuncGetAttributes(&fa, k_gram_tc<true>));
      launch_regs = fa.numRegs;
    }
    if (launch_regs < kLaunchRegs)
      throw MgError(MG_ERR_CUDA, "fused tensor-core sampler built with too few registers");
    if (p.retry_work == nullptr)
      throw MgError(MG_ERR_STATE, "fused tensor-core sampler without its retry work area");
    k_gram_tc<true><<<num_sms, kTcThreadsFused, smem, s>>>(p, nullptr);
    MG_CUDA(cudaGetLastError());
    if (mid) MG_CUDA(cudaEventRecord(mid, s));
    if (nsplit > 0) {
      k_sum_parts<<<(nsplit + 7) / 8, 256, 0, s>>>(p.scratch, split_rows, nsplit, gram, 1);
      MG_CUDA(cudaGetLastError());
      const int blocks = std::min(num_sms * 2, (nsplit + 4 * kFinWarps - 1) / (4 * kFinWarps));
      k_finish_tc<<<blocks, kFinWarps * 32, kFinSmem, s>>>(p, gram, split_rows, nsplit);
      MG_CUDA(cudaGetLastError());
    }
    return true;
  }
  launch_gram_tc(p, gram, split_rows, nsplit, KP, s, num_sms, mid);
  if (p.one)
    k_finish_one_tc<<<num_sms * 8, 256, 0, s>>>(p, gram);
  else
    k_finish_tc<<<num_sms * 2, kFinWarps * 32, kFinSmem, s>>>(p, gram, nullptr, 0);
  MG_CUDA(cudaGetLastError());
  return true;
}

}  // namespace mg
