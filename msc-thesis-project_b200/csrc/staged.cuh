// staged.cuh -- full decompression of 64-bit-lane columns (u64 FFOR / BP,
// f64 ALP) with each vector's packed words staged in shared memory.
//
// The register-held decode (k_store) waits for a vector's packed words
// before it can unpack them, and at 64-bit widths it cannot hold the next
// vector's words as well.  Here every warp owns two shared-memory slots of
// 4 KiB (the packed words of one vector of width <= 32): while vector i is
// unpacked from slot i % 2, a bulk copy (cp.async.bulk, completion counted
// on the slot's mbarrier) brings vector i + 1 into the other slot, and the
// copy of vector i + 2 is issued as soon as vector i's slot is read.  The
// unpack reads each value's one or two 32-bit stream words straight from
// the slot.  Vectors wider than 32 bits, or with a packed-word address that
// is not 16-byte aligned, take the register-held decode of k_store's
// register-capped variant.
//
// Every wait on an mbarrier is bounded (about a second of SM clocks); a
// wait that gives up raises FLSGPU_WAIT_TIMEOUT in the status word, waits
// (bounded) for the warp's other copy in flight, and ends the warp's work.
#pragma once

#include "kernels.cuh"

namespace flsb200 {

constexpr int kStageSlotBytes = 4096;  // 32 lines of 128 B: widths up to 32
constexpr int kStageMaxW = 32;
constexpr long long kStageWaitCycles = 2000000000ll;  // ~1 s at 1.965 GHz

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
}

// bytes (a multiple of 16) from 16-byte-aligned global src to the slot;
// completion counted on bar (one arrival with the expected byte count)
__device__ __forceinline__ void bulk_to_slot(void *dst, const void *src, uint32_t bytes,
                                             uint64_t *bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

// Waits for the completion of bar's phase with parity ph; false when about
// a second of SM clocks passed first.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t ph) {
  const uint32_t a = smem_addr(bar);
  const long long t0 = clock64();
  while (true) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(a), "r"(ph)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > kStageWaitCycles) return false;
  }
}

// Decodes the thread's 32 values of a vector whose packed 64-bit lines
// start at p32 (as 32-bit words; shared memory when SMEM, else global):
// thread t = half t / 16 of lane t % 16; 32-bit stream word j of the half
// is at (j odd ? pb : pa)[16 j] (the layout of the 64-bit lines: word m of
// lane l at 32 (m / 2) + 2 l + m % 2).  Each value reads the one to three
// words it spans when it is decoded, so few registers are live.
template <bool SMEM, int VAR, class X, class Put>
__device__ __forceinline__ void decode_words64(const uint32_t *base, int w, int t, const X &xf,
                                               Put &&put) {
  const int lane = t & 15, half = t >> 4;
  switch_width64(w, [&](auto wc) {
    constexpr int W = decltype(wc)::value;
    constexpr int P = policy_of<uint64_t, VAR>(W);
    const int oddm0 = half & W & 1;
    const uint32_t *p32 = base + 2 * lane + half * 16 * W;
    const uint32_t *pa = p32 - (oddm0 ? 15 : 0);
    const uint32_t *pb = p32 - (oddm0 ? 0 : 15);
    auto ld = [&](int j) -> uint32_t {
      const uint32_t *q = ((j & 1) ? pb : pa) + 16 * j;
      if constexpr (SMEM)
        return *q;
      else
        return __ldg(q);
    };
#pragma unroll
    for (int k = 0; k < 32; ++k) {
      uint64_t v = 0;
      if (W > 0) {
        const int bit = k * W, j = bit >> 5, o = bit & 31;
        const int je = (bit + W - 1) >> 5;
        const uint32_t x0 = ld(j);
        const uint32_t x1 = (je >= j + 1) ? ld(j + 1) : 0u;
        const uint32_t x2 = (je >= j + 2) ? ld(j + 2) : 0u;
        const uint32_t lo = o ? funnel_r(x0, x1, (uint32_t)o) : x0;
        uint32_t hi = 0;
        if (W > 32 - o) hi = o ? funnel_r(x1, x2, (uint32_t)o) : x1;
        v = (((uint64_t)hi << 32) | lo) & mask64<W>();
      }
      put(lane + 16 * (32 * half + k), xf(v), IntC<P>{});
    }
  });
}

// The first 32 exceptions of a vector (lane i: position and value of
// exception i; position VEC on lanes past the count), and the vector's
// exception count.  Loaded one vector ahead of the decode.
template <typename T, int KIND>
__device__ __forceinline__ uint32_t first_exceptions(const ColumnParams &c, const Meta<T> &m, int t,
                                                     uint32_t &p0, T &e0) {
  p0 = VEC;
  e0 = T(0);
  uint32_t ecnt = 0;
  if constexpr (KIND == K_ALP || KIND == K_ALPX) {
    const bool pre = (KIND == K_ALP && c.patch && c.counts) || (KIND == K_ALPX && c.patch && c.oc);
    if constexpr (KIND == K_ALP)
      ecnt = m.ecnt;
    else
      ecnt = __reduce_add_sync(0xffffffffu, m.ecnt >> 10) & 0xFFFFu;
    if (pre && (uint32_t)t < ecnt) {
      p0 = c.pos[m.eo + t];
      e0 = reinterpret_cast<const T *>(c.exc)[m.eo + t];
    }
  }
  return ecnt;
}

// One vector: decode (from the slot when s32 is given, else from global
// memory), then patch its exceptions (ALP columns; p0 / e0 / ecnt from
// first_exceptions); as store_one.
template <typename T, int KIND, int VAR>
__device__ __forceinline__ void store_one_staged(const KernelParams &p, size_t vi, const Meta<T> &m,
                                                 int t, const uint32_t *s32, uint32_t p0, T e0,
                                                 uint32_t ecnt) {
  using U = typename UintOf<T>::U;
  using X = typename XformOf<T, KIND>::type;
  const ColumnParams &c = p.c;
  const U *vin;
  int w;
  X xf;
  if (!setup_from_meta<T, KIND>(c, p.d_status, m, t, vin, w, xf)) return;
  const size_t vbase = vi * VEC;
  const size_t rem = c.n_values - vbase;
  const int lim = rem < (size_t)VEC ? (int)rem : VEC;
  T *out = reinterpret_cast<T *>(p.out) + vbase;
  [[maybe_unused]] const bool pre =
      (KIND == K_ALP && c.patch && c.counts) || (KIND == K_ALPX && c.patch && c.oc);
  auto put_full = [&](int idx, T v, auto pc) { store_out<T, decltype(pc)::value>(out + idx, v); };
  auto put_lim = [&](int idx, T v, auto pc) {
    if (idx < lim) store_out<T, decltype(pc)::value>(out + idx, v);
  };
  if (s32) {
    if (lim == VEC)
      decode_words64<true, VAR>(s32, w, t, xf, put_full);
    else
      decode_words64<true, VAR>(s32, w, t, xf, put_lim);
  } else {
    if (lim == VEC)
      decode_values<T, VAR>(vin, w, t, xf, put_full);
    else
      decode_values<T, VAR>(vin, w, t, xf, put_lim);
  }
  if constexpr (KIND == K_ALP || KIND == K_ALPX) {
    if (pre) {
      __syncwarp();
      bool bad = (uint32_t)t < ecnt && p0 >= VEC;
      if ((int)p0 < lim) out[p0] = e0;
      const T *exc = reinterpret_cast<const T *>(c.exc);
      bad |= patch_batched<T>(c.pos + m.eo, exc + m.eo, 32, ecnt, t, [&](uint32_t ps, T e) {
        if ((int)ps < lim) out[ps] = e;
      });
      if (__any_sync(0xffffffffu, bad) && t == 0) flag_status(p.d_status, FLSGPU_BAD_EXCEPTION);
    } else if (c.patch) {
      __syncwarp();
      patch_vector<T, KIND>(c, p.d_status, vi, t, [&](int ps, T e) {
        if (ps < lim) out[ps] = e;
      });
    }
  }
}

// Whether vector metadata m is decoded from a slot: width 1..32, metadata
// that passes the checks, packed words 16-byte aligned.
template <typename T, int KIND>
__device__ __forceinline__ bool stageable(const ColumnParams &c, const Meta<T> &m) {
  if (m.w < 1 || m.w > kStageMaxW) return false;
  if (c.n_packed && (m.off > c.n_packed || (size_t)m.w * 16 > c.n_packed - m.off)) return false;
  if constexpr (std::is_same<T, double>::value) {
    if (m.fi > 18 || m.ei > 20) return false;
  }
  const uintptr_t src = reinterpret_cast<uintptr_t>(c.packed) + m.off * 8;
  return (src & 15u) == 0;
}

template <typename T, int KIND>
__global__ void __launch_bounds__(256, 2) k_store_staged(const KernelParams p) {
  static_assert(sizeof(T) == 8, "64-bit lanes only");
  constexpr int VAR = VAR_AUTO | VAR_OCC;
  extern __shared__ __align__(128) unsigned char st_smem[];
  const int t = threadIdx.x & 31, wib = threadIdx.x >> 5;
  unsigned char *slot_base = st_smem + (size_t)wib * 2 * kStageSlotBytes;
  uint64_t *bars = reinterpret_cast<uint64_t *>(st_smem + 8 * 2 * kStageSlotBytes) + 2 * wib;
  if (t == 0) {
    mbar_init(&bars[0]);
    mbar_init(&bars[1]);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncwarp();
  const ColumnParams &c = p.c;
  const size_t n = c.n_vecs;
  const size_t gw = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
  const char *packed = reinterpret_cast<const char *>(c.packed);
  auto issue = [&](const Meta<T> &m, int s) {
    if (t == 0)
      bulk_to_slot(slot_base + s * kStageSlotBytes, packed + m.off * 8, (uint32_t)m.w * 128u,
                   &bars[s]);
  };
  // metadata of the warp's vectors i, i + 1, i + 2 (loads one step ahead)
  Meta<T> m0{}, m1{}, m2{};
  bool st0 = false, st1 = false;
  if (gw < n) {
    m0 = load_meta<T, KIND>(c, gw, t);
    st0 = stageable<T, KIND>(c, m0);
    if (st0) issue(m0, 0);
  }
  if (gw + nw < n) {
    m1 = load_meta<T, KIND>(c, gw + nw, t);
    st1 = stageable<T, KIND>(c, m1);
    if (st1) issue(m1, 1);
  }
  uint32_t phase = 0;  // bit s: parity of slot s's next completion
  int s = 0;
  // the first exceptions of the warp's next vector
  uint32_t xp = VEC, xc = 0;
  T xe = T(0);
  if (gw < n) xc = first_exceptions<T, KIND>(c, m0, t, xp, xe);
  for (size_t vi = gw; vi < n; vi += nw, s ^= 1) {
    const bool has2 = vi + 2 * nw < n;
    if (has2) m2 = load_meta<T, KIND>(c, vi + 2 * nw, t);
    const uint32_t cp = xp, cc = xc;
    const T ce = xe;
    if (vi + nw < n) xc = first_exceptions<T, KIND>(c, m1, t, xp, xe);
    const uint32_t *s32 = nullptr;
    if (st0) {
      // the decision to give up is the warp's, so that it stays converged
      if (!__all_sync(0xffffffffu, mbar_wait(&bars[s], (phase >> s) & 1u))) {
        if (t == 0) flag_status(p.d_status, FLSGPU_WAIT_TIMEOUT);
        // the other slot's copy may still be in flight: wait for it before
        // the warp stops using its slots
        if (st1) mbar_wait(&bars[s ^ 1], (phase >> (s ^ 1)) & 1u);
        return;
      }
      phase ^= 1u << s;
      s32 = reinterpret_cast<const uint32_t *>(slot_base + s * kStageSlotBytes);
    }
    store_one_staged<T, KIND, VAR>(p, vi, m0, t, s32, cp, ce, cc);
    bool st2 = false;
    if (has2) {
      st2 = stageable<T, KIND>(c, m2);
      if (st2) {
        // the slot's reads are done before the bulk copy overwrites it
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncwarp();
        issue(m2, s);
      }
    }
    m0 = m1;
    st0 = st1;
    m1 = m2;
    st1 = st2;
  }
}

template <typename T, int KIND>
flsgpu_status launch_staged(const KernelParams &p, cudaStream_t s) {
  constexpr size_t smem = (size_t)8 * 2 * kStageSlotBytes + 8 * 2 * sizeof(uint64_t);
  static int bps = 0;
  if (bps == 0) {
    cudaFuncSetAttribute(k_store_staged<T, KIND>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
    int b = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_store_staged<T, KIND>, 256, smem);
    bps = b > 0 ? b : 1;
  }
  const unsigned grid = persistent_blocks(p.c.n_vecs, 8, bps);
  k_store_staged<T, KIND><<<grid, 256, smem, s>>>(p);
  note_launch();
  return check_cuda(cudaGetLastError(), "staged decode launch");
}

}  // namespace flsb200
