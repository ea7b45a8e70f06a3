// Gram matrices of the LLR blocks on the 5th-generation tensor cores (tcgen05).
//
// For a Casorati block C (m x n complex) let D = [Re C | Im C] (m x 2n real).  Then
// P = D^T D (2n x 2n) gives G = C^H C as
//   Re G[i][j] = P[i][j] + P[n+i][n+j],   Im G[i][j] = P[i][n+j] - P[n+i][j].
// P is one 128 x 128 UMMA accumulator in tensor memory (2n <= 128), K = the m voxel rows.
// Both operands are the same shared-memory tile of D in the K-major layout with the 128-byte
// swizzle (one 128-byte row of 32 TF32 per column of D and chunk), so A = B and the MMA
// computes D^T D directly.
// Precision: 3xTF32 -- x = hi + lo with hi = tf32(x), and P accumulates hi*hi + hi*lo + lo*hi
// in FP32, which keeps FP32-level accuracy (the lo*lo term is below FP32 rounding).
// Rows stream in 32-row chunks, double-buffered, with the loads of the chunk two positions
// ahead (possibly of the CTA's next block) in flight: while the tensor core consumes one chunk
// the 8 warps gather, phase-correct and split the next one.  One elected thread issues the
// MMAs and commits them to an mbarrier; every wait is bounded and reports a timeout through
// op.err instead of hanging.
#include <cstdio>
#include <algorithm>

#include "llr_prox_common.cuh"
#include "llr_umma.cuh"

namespace llr {

namespace {

constexpr int kTcWarps = 8;
constexpr int kTcThreads = 32 * kTcWarps;
constexpr int kKC = 32;                    // rows (K) per staged chunk
constexpr int kQT = (64 + kTcWarps - 1) / kTcWarps;   // volumes per warp per chunk (kTcWarps x kQT >= n)
constexpr int kOpBytes = 128 * kKC * 4;    // one operand plane (hi or lo) of one chunk
// Row table of one block: planar offset of every row and either the row's phase (uniform
// over the volumes) or its coordinates (per-volume phase).  The kernel keeps kRowBufs tables:
// the one of the block being converted and those of the blocks whose chunks are prefetched.
union TcRowAux {
  float2 ph;
  int2 c;              // x, y | z << 16
};

struct TcLayout {
  size_t off_hdr, off_row, off_aux, off_op, total;
  int op_bytes;        // bytes of the operand / P-staging region
  int nbuf;            // row tables: 2 (3 when a block is a single chunk)
};

struct TcHdr {
  unsigned long long mbar[3];   // chunk buffer 0, chunk buffer 1, block done
  unsigned int tmem;            // tensor-memory base address
  int shift[3];
  int fail;
  int pad;
};

// Instruction descriptor: TF32 x TF32 -> F32, both K-major, M = 128, N = 128.
constexpr uint32_t kIdesc = umma_idesc_tf32(128, 128);

template <int NPMAX>
__global__ void __launch_bounds__(kTcThreads, 3) llr_gram_tc_kernel(BlockSource src, ProxOp op, TcLayout L) {
  extern __shared__ __align__(1024) unsigned char smem[];
  TcHdr* hdr = reinterpret_cast<TcHdr*>(smem + L.off_hdr);
  int* row_off = reinterpret_cast<int*>(smem + L.off_row);        // [nbuf][m]
  TcRowAux* row_aux = reinterpret_cast<TcRowAux*>(smem + L.off_aux);   // [nbuf][m]
  unsigned char* ops = smem + L.off_op;   // [buf][hi, lo] planes; reused as P staging
  const int m = op.m, n = op.n, tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long long qstride = src.kind == 1 ? src.g.V : (long long)m;
  const int nchunks = (m + kKC - 1) / kKC;
  const int nbuf = L.nbuf, la = nbuf - 1;   // row-table lookahead in blocks

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&hdr->tmem)),
                 "r"(128u));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int b = 0; b < 3; ++b)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&hdr->mbar[b])));
    asm volatile("fence.mbarrier_init.release.cluster;");
    block_shift(src, hdr->shift);
    hdr->fail = 0;
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = hdr->tmem;
  const int sh[3] = {hdr->shift[0], hdr->shift[1], hdr->shift[2]};
  uint32_t phase[3] = {0u, 0u, 0u};
  bool used[2] = {false, false};
  bool failed = false;

  // Lane layout of the gather: lane = row of the chunk, warp w = volumes w, w + kTcWarps, ...: every
  // request reads 32 consecutive rows of one volume (the block's runs along y of one DRAM
  // page); requests that mix volumes, one short run each, reach a fraction of the HBM rate.
  // In shared memory the 32 lanes write one 128-byte swizzled row (all banks).
  // Chunks form one stream over the CTA's blocks; two register sets alternate, and after a
  // set is converted it is refilled with the chunk two positions ahead, so two chunks of
  // loads are in flight while the tensor core and the epilogue run.
  float2 preA[kQT], preB[kQT];
  auto build_rows = [&](long long b, int buf) {
    int* ro = row_off + (size_t)buf * m;
    TcRowAux* ra = row_aux + (size_t)buf * m;
    for (int r = tid; r < m; r += kTcThreads) {
      if (src.kind == 1) {
        int ix, iy, iz;
        block_row_coord(src, b, sh, r, ix, iy, iz);
        ro[r] = (int)planar_index(src.g, ix, iy, iz, 0);
        TcRowAux a;
        if (src.ph_uniform) a.ph = phase_at(src.ph, src.g, 0, ix, iy, iz);
        else a.c = make_int2(ix, iy | (iz << 16));
        ra[r] = a;
      } else {
        ro[r] = r;
      }
    }
  };
  auto block_base = [&](long long b) { return src.kind == 1 ? 0ll : b * (long long)m * n; };
  auto load_chunk = [&](float2 (&pre)[kQT], int c, long long b, int buf) {
    const int r = c * kKC + lane;
    const int ro = r < m ? row_off[(size_t)buf * m + r] : -1;
    const float2* rowp = src.data + block_base(b) + (ro >= 0 ? ro : 0);
#pragma unroll
    for (int t = 0; t < kQT; ++t) {
      const int q = warp + kTcWarps * t;
      pre[t] = (q < n && ro >= 0) ? rowp[(long long)q * qstride] : make_float2(0.f, 0.f);
    }
  };
  // the chunk `ahead` positions after (block iteration j, chunk c); false past the CTA's blocks
  auto locate = [&](long long blk, int j, int c, int ahead, long long& b2, int& j2, int& c2) {
    c2 = c + ahead;
    j2 = j;
    b2 = blk;
    while (c2 >= nchunks) { c2 -= nchunks; ++j2; b2 += gridDim.x; }
    return b2 < src.nblocks;
  };
  // one chunk: wait for its operand buffer, convert `pre` into it, refill `pre` two chunks
  // ahead, hand the buffer to the tensor core
  int gpar = 0;
  // operand offsets of this thread's elements: row q = warp + kTcWarps t (and n + q), column
  // lane; adding 8 to a row leaves its swizzle phase and moves it one 1 KB atom on, so
  // op_offset(q + 8 t, lane) = op_offset(q, lane) + 1024 t
  static_assert(kTcWarps == 8, "the 1 KB step per t assumes rows 8 apart");
  const int oq0 = op_offset(warp, lane), oi0 = op_offset(n + warp, lane);
  auto step = [&](float2 (&pre)[kQT], long long blk, int j, int c) -> bool {
    const int b = gpar;
    if (used[b]) {  // the MMAs that read this buffer two chunks ago must be done
      const bool ok = mbar_wait(smem_u32(&hdr->mbar[b]), phase[b]);
      phase[b] ^= 1u;
      if (__syncthreads_or(!ok)) return false;
    }
    unsigned char* hi = ops + (size_t)b * 2 * kOpBytes;
    unsigned char* lo = hi + kOpBytes;
    const int r = c * kKC + lane;
    const TcRowAux* ra = row_aux + (size_t)(j % nbuf) * m;
    const bool ph_row = src.kind == 1 && r < m;
    float2 p = make_float2(1.f, 0.f);
    if (ph_row && src.ph_uniform) p = ra[r].ph;
#pragma unroll
    for (int t = 0; t < kQT; ++t) {
      const int q = warp + kTcWarps * t;
      if (q >= n) break;                              // warp-uniform
      float2 x = pre[t];
      if (ph_row) {
        if (!src.ph_uniform) {
          const int2 cc = ra[r].c;
          p = phase_at(src.ph, src.g, q, cc.x, cc.y & 0xffff, cc.y >> 16);
        }
        x = cscale(cmul_bc(x, p), src.load_scale);
      }
      const uint32_t a = tf32_rna(x.x), bb = tf32_rna(x.y);
      const int oq = oq0 + 1024 * t, oi = oi0 + 1024 * t;
      *reinterpret_cast<uint32_t*>(hi + oq) = a;
      *reinterpret_cast<uint32_t*>(hi + oi) = bb;
      *reinterpret_cast<uint32_t*>(lo + oq) = __float_as_uint(x.x - __uint_as_float(a));
      *reinterpret_cast<uint32_t*>(lo + oi) = __float_as_uint(x.y - __uint_as_float(bb));
    }
    {
      long long b2;
      int j2, c2;
      if (locate(blk, j, c, 2, b2, j2, c2)) load_chunk(pre, c2, b2, j2 % nbuf);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;");
      const uint32_t ah = smem_u32(hi), al = smem_u32(lo);
#pragma unroll
      for (int s = 0; s < kKC / 8; ++s) {
        const uint64_t dh = umma_desc_sw128(ah + s * 32);
        const uint64_t dl = umma_desc_sw128(al + s * 32);
        umma_tf32(tmem, dh, dh, kIdesc, (c > 0 || s > 0) ? 1u : 0u);
        umma_tf32(tmem, dh, dl, kIdesc, 1u);
        umma_tf32(tmem, dl, dh, kIdesc, 1u);
      }
      umma_commit(smem_u32(&hdr->mbar[b]));
      if (c == nchunks - 1) umma_commit(smem_u32(&hdr->mbar[2]));
    }
    used[b] = true;
    gpar ^= 1;
    return true;
  };

  // operand planes start zeroed: rows 2n..127 (M padding) are never written by the gather
  for (int i = tid; i < 4 * kOpBytes / 16; i += kTcThreads)
    reinterpret_cast<float4*>(ops)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
  long long blk = blockIdx.x;
  if (blk < src.nblocks) {
    for (int jj = 0; jj <= la; ++jj)
      if (blk + (long long)jj * gridDim.x < src.nblocks) build_rows(blk + (long long)jj * gridDim.x, jj % nbuf);
    __syncthreads();
    long long b2;
    int j2, c2;
    if (locate(blk, 0, 0, 0, b2, j2, c2)) load_chunk(preA, c2, b2, j2 % nbuf);
    if (locate(blk, 0, 0, 1, b2, j2, c2)) load_chunk(preB, c2, b2, j2 % nbuf);
  }

  for (int j = 0; blk < src.nblocks && !failed; blk += gridDim.x, ++j) {
    if (j > 0) {   // the table of the block `la` ahead goes into the buffer the previous block freed
      const long long bl = blk + (long long)la * gridDim.x;
      if (bl < src.nblocks) build_rows(bl, (j + la) % nbuf);
      __syncthreads();
    }
    for (int c = 0; c < nchunks; ++c) {
      const bool ok = gpar == 0 ? step(preA, blk, j, c) : step(preB, blk, j, c);
      if (!ok) { failed = true; break; }
    }
    if (failed) break;
    // all MMAs of this block complete -> read P and stage it in the (now idle) operand area
    {
      const bool ok = mbar_wait(smem_u32(&hdr->mbar[2]), phase[2]);
      phase[2] ^= 1u;
      // the done barrier implies every chunk barrier's MMAs finished too; consume them
      for (int bb = 0; bb < 2; ++bb)
        if (used[bb]) {
          mbar_wait(smem_u32(&hdr->mbar[bb]), phase[bb]);
          phase[bb] ^= 1u;
          used[bb] = false;
        }
      if (__syncthreads_or(!ok)) { failed = true; break; }
    }
    asm volatile("tcgen05.fence::after_thread_sync;");
    float* Ps = reinterpret_cast<float*>(ops);
    const int ldp = 2 * n + 1;
    // warp w reads TMEM lanes 32 (w mod 4) .. + 31 (its quadrant); the warps sharing a quadrant
    // split the 32-column chunks
    const int quad = warp & 3;
    const int a = 32 * quad + lane;          // accumulator row held by this thread
    for (int cc = 32 * (warp >> 2); cc < 2 * n; cc += 32 * (kTcWarps / 4)) {
      uint32_t r[32];
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
          "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
            "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
            "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
            "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
          : "r"(tmem + ((uint32_t)(32 * quad) << 16) + (uint32_t)cc));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (a < 2 * n) {
#pragma unroll
        for (int jj = 0; jj < 32; ++jj)
          if (cc + jj < 2 * n) Ps[a * ldp + cc + jj] = __uint_as_float(r[jj]);
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    // packed lower triangle by row pairs (i, n - 1 - i): n + 1 elements per pair, so a warp's
    // lanes stay busy; two elements per lane in flight
    float2* G = op.gram + blk * op.gram_stride;
    for (int i = warp; i < (n + 1) / 2; i += kTcThreads / 32) {
      const int i2 = n - 1 - i, len = i2 == i ? i + 1 : n + 1;
      for (int s0 = lane; s0 < len; s0 += 64) {
        float re[2], im[2];
        int row[2], col[2];
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          const int s = min(s0 + 32 * u, len - 1);
          row[u] = s <= i ? i : i2;
          col[u] = s <= i ? s : s - i - 1;
          re[u] = Ps[row[u] * ldp + col[u]] + Ps[(n + row[u]) * ldp + n + col[u]];
          im[u] = Ps[row[u] * ldp + n + col[u]] - Ps[(n + row[u]) * ldp + col[u]];
        }
#pragma unroll
        for (int u = 0; u < 2; ++u)
          if (s0 + 32 * u < len) G[(long long)row[u] * (row[u] + 1) / 2 + col[u]] = make_float2(re[u], im[u]);
      }
    }
    __syncthreads();
    // the staging overwrote the padding rows 2n..127 of the operand planes: zero them again
    for (int i = tid; i < 4 * (128 - 2 * n) * 8; i += kTcThreads) {   // 8 x 16 B per 128-B row
      const int plane = i / ((128 - 2 * n) * 8), rem = i - plane * ((128 - 2 * n) * 8);
      const int mn = 2 * n + (rem >> 3), c16 = rem & 7;
      *reinterpret_cast<float4*>(ops + (size_t)plane * kOpBytes + (mn >> 3) * 1024 + (mn & 7) * 128 + c16 * 16) =
          make_float4(0.f, 0.f, 0.f, 0.f);
    }
    __syncthreads();
  }

  if (failed && tid == 0 && op.err) atomicExch(op.err, 1);
  // make sure nothing is still writing the accumulator before it is released
  if (tid == 0) {
    umma_commit(smem_u32(&hdr->mbar[2]));
  }
  mbar_wait(smem_u32(&hdr->mbar[2]), phase[2]);
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128u));
}

template <int NPMAX>
TcLayout make_tc_layout(int m, int n) {
  TcLayout L;
  size_t off = 0;
  L.off_hdr = off; off = align16(off + sizeof(TcHdr));
  L.nbuf = m <= kKC ? 3 : 2;
  L.off_row = off; off = align16(off + sizeof(int) * (size_t)m * L.nbuf);
  L.off_aux = off; off = align16(off + sizeof(TcRowAux) * (size_t)m * L.nbuf);
  off = (off + 1023) & ~size_t(1023);
  L.off_op = off;
  const size_t opb = std::max<size_t>(4 * (size_t)kOpBytes, sizeof(float) * (size_t)(2 * n) * (2 * n + 1));
  L.op_bytes = (int)opb;
  off += opb;
  L.total = off;
  return L;
}

}  // namespace

bool llr_gram_tc_supported(int m, int n) {
  if (n < 1 || 2 * n > 128 || m < 1 || 8 * n > 4 * kTcThreads) return false;
  return make_tc_layout<64>(m, n).total <= 227 * 1024;
}

int launch_llr_gram_tc(const BlockSource& src, const ProxOp& op, cudaStream_t stream) {
  if (2 * op.n > 128) return set_error(LLR_ERR_UNSUPPORTED, "tensor-core Gram needs 2n <= 128 (n = %d)", op.n);
  TcLayout L = make_tc_layout<64>(op.m, op.n);
  if (L.total > 227 * 1024) return set_error(LLR_ERR_UNSUPPORTED, "tensor-core Gram needs %zu B smem", L.total);
  auto kern = llr_gram_tc_kernel<64>;
  LLR_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.total));
  LLR_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
  int dev = 0, nsm = 0, smem_sm = 0, regs_sm = 0;
  LLR_CUDA_TRY(cudaGetDevice(&dev));
  LLR_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  LLR_CUDA_TRY(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
  LLR_CUDA_TRY(cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev));
  cudaFuncAttributes fa{};
  LLR_CUDA_TRY(cudaFuncGetAttributes(&fa, kern));
  // Residency from the kernel's own resources. The occupancy query reports one CTA per SM for
  // this kernel although three fit, so the count is derived here: shared memory (the driver
  // reserves 1 KB per CTA), registers (allocated per warp in units of 256) and TMEM (128 of
  // the SM's 512 columns per CTA). The kernel strides over blocks, so a grid larger than
  // what is resident is still correct, only slower.
  const int regs_warp = ((fa.numRegs * 32 + 255) / 256) * 256;
  const int by_regs = regs_warp > 0 ? regs_sm / (regs_warp * (kTcThreads / 32)) : 4;
  const int by_smem = smem_sm / (int)(L.total + fa.sharedSizeBytes + 1024);
  int occ = std::min(std::min(by_regs, by_smem), 4);
  if (occ < 1) return set_error(LLR_ERR_UNSUPPORTED, "tensor-core Gram kernel cannot be resident");
  const long long grid = std::min<long long>(src.nblocks, (long long)nsm * occ);
  if (grid < 1) return LLR_OK;
  note_launch();
  kern<<<(unsigned)grid, kTcThreads, L.total, stream>>>(src, op, L);
  LLR_CUDA_TRY(cudaGetLastError());
  return LLR_OK;
}

}  // namespace llr
