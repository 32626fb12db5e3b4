// Warp-specialised pipelined step kernels (sm_100a).
//
// One persistent CTA per SM walks a contiguous range of patches.  The first W
// warps are producers: for every patch they read the patch's copy descriptors
// (built on the host, rows of one source array coalesced into runs) and copy
// them into the next free stage of an n-stage ring in shared memory, either as one
// TMA bulk copy (cp.async.bulk global -> shared) per descriptor completing on
// the stage's "full" mbarrier by transaction count, or as 16-byte cp.async
// pieces spread over the warp's lanes, completing by one cp.async arrival per
// lane.  The first descriptor of every patch copies the patch's table blob
// (local row indices into the stage, metric factors, reconstruction rows, slot
// tables), so the compute warps make no dependent global loads: they wait on
// "full", run the same per-run arithmetic as the direct kernels from shared
// memory, write their outputs straight to global memory and release the stage
// on its "empty" mbarrier (one arrival per compute warp).
//
// Every wait is bounded by the global timer.  A wait that runs out sets bit 0
// of the device status word and a CTA-wide abort flag; the other waits then
// return at once, compute is skipped, and the producers wait (again bounded)
// for the copies they issued before the CTA exits.  Sources are this GPU's
// global memory only; no copy uses cluster multicast.
#pragma once

#include "step_kernels.cuh"

namespace ifdtd {
namespace pipe {

constexpr int kMaxStages = 8;
constexpr int kDescPerLane = 4;
constexpr int kMaxDesc = 32 * kDescPerLane;  // copy descriptors per patch
constexpr int kMaxThreads = 384;             // producer warps + compute warps
// Registers are granted to warps in groups of four: 12 warps x 32 x 168 <= 65536.
constexpr int kMaxRegs = 168;
// Wide E-phase CTAs: up to 20 warps at 96 registers (20 x 32 x 96 <= 65536);
// the E consumer fits 96 registers without spilling, the H consumer does not.
constexpr int kWideRegs = 96;
constexpr int kWideMaxThreads = 640;
constexpr uint64_t kWaitNs = 500ull * 1000 * 1000;  // bound of one wait (0.5 s)

// Descriptor sources (int4 {src, first row, stage byte offset, bytes}).
enum Src : int { kSrcEr = 0, kSrcEt = 1, kSrcHt = 2, kSrcHr = 3, kSrcJsum = 4, kSrcTab = 5, kSrcSi = 6, kSrcJ0 = 8 };

// H-phase blob header (ints; offsets are bytes from the stage start).
enum KhHead : int {
  kh_ea, kh_ne, kh_fa, kh_nf, kh_o_er, kh_o_et, kh_o_ht, kh_o_hr, kh_o_J,
  kh_o_eloc, kh_o_einv, kh_o_floc, kh_o_fw, kh_o_fpl, kh_o_si, kh_o_esis, kh_o_hnew, kh_head_ints = 20
};
// E-phase blob header.
enum KeHead : int {
  ke_nv, ke_ea, ke_ne, ke_o_ht, ke_o_hr, ke_o_J, ke_o_er, ke_o_et, ke_o_vid, ke_o_vh,
  ke_o_vj, ke_o_vcoef, ke_o_vwc, ke_o_eloc, ke_o_einv, ke_o_etan, ke_o_end, ke_src, ke_head_ints = 20
};
// ke_o_end: the end of the staged rows (the stage holds nothing after them).
// ke_src: bit 0 = an owned vertex carries a vertical source support, bit 1 =
// an owned edge carries a tangential one (other patches skip the search).

// Bytes of per-layer rows at the start of dynamic shared memory (host and
// device), rounded to 128 so the stages start aligned.
__host__ __device__ inline int layer_block_bytes(int layer_reals, int real_bytes) {
  return (layer_reals * real_bytes + 127) / 128 * 128;
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_inval(uint64_t* bar) {
  asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 16-byte asynchronous copy global -> shared (L2 only), and the arrival on an
// mbarrier that fires once all of this thread's earlier cp.async copies have
// landed (.noinc: the arrival is one of the barrier's expected arrivals).
__device__ __forceinline__ void cp16_async(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_arrive_noinc(uint64_t* bar) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Bounded wait for the phase of `bar` with the given parity.  abort_flag ==
// nullptr: ignore the CTA abort flag (used while draining).
__device__ __forceinline__ bool wait_phase(uint64_t* bar, uint32_t parity, volatile int* abort_flag, int* status) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  for (uint32_t i = 1; i < (1u << 30); ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((i & 15u) == 0) {
      if (abort_flag && *abort_flag) return false;
      if (global_ns() - t0 > kWaitNs) break;
    }
  }
  if (abort_flag) *abort_flag = 1;
  atomicOr(status, 1);
  return false;
}

struct Ring {
  unsigned char* stages;
  int stage_bytes, n_stages;
  uint64_t *full, *empty;
  volatile int* abort_flag;
  int* status;
};

template <typename real>
__device__ __forceinline__ const void* desc_source(const Rec<real>& R, const unsigned char* tab, int src, int row) {
  const size_t r = (size_t)row;
  switch (src) {
    case kSrcEr: return R.er + r * R.Pn;
    case kSrcEt: return R.et + r * R.Pm;
    case kSrcHt: return R.ht + r * R.Pn;
    case kSrcHr: return R.hr + r * R.Pm;
    case kSrcJsum: return jsum(R) + r * 3 * R.Pm;
    case kSrcTab: return tab + r * 16;
    case kSrcSi: return R.si_mem + r * R.si_terms;
    default: return R.J[(src - kSrcJ0) & (kMaxSpecies - 1)] + r * 3 * R.Pm;
  }
}

// Producer warp w of W: fills stage i % n_stages with its share (descriptors
// w, w + W, ...) of patch p0 + i; a single warp issuing lane-parallel bulk
// copies is issue-bound, so W warps split the descriptor list.  Descriptor
// offsets (dptr) are read 32 patches at a time and each patch's descriptors
// one patch ahead, so their latency overlaps the wait for a free stage.
// COPY 0: one TMA bulk copy per descriptor, completion by transaction count
// on the stage's full barrier (one expect_tx arrival per producer warp).
// COPY 1: 16-byte cp.async pieces, lane-parallel within each descriptor,
// completion by one cp.async arrival per producer lane.
template <int COPY, typename real>
__device__ void produce(const Rec<real>& R, const Ring& G, int p0, int p1, int n_patches, const int* dptr,
                        const int4* desc, const unsigned char* tab, int w, int W) {
  const int lane = threadIdx.x & 31;
  int win = p0;
  int dpw = __ldg(dptr + min(win + lane, n_patches));
  int4 cur[kDescPerLane], nxt[kDescPerLane];
  int ncur = 0, nnxt = 0;
  auto fetch = [&](int p, int4* d, int& n) {
    if (p + 1 - win >= 32) {
      win = p;
      dpw = __ldg(dptr + min(win + lane, n_patches));
    }
    const int b = __shfl_sync(0xFFFFFFFFu, dpw, p - win);
    n = __shfl_sync(0xFFFFFFFFu, dpw, p + 1 - win) - b;
#pragma unroll
    for (int k = 0; k < kDescPerLane; ++k) {
      const int j = w + W * (lane + 32 * k);
      d[k] = j < n ? __ldg(desc + b + j) : make_int4(0, 0, 0, 0);
    }
  };
  if (p0 < p1) fetch(p0, cur, ncur);
  int i = 0;
  bool ok = true;
  for (int p = p0; p < p1; ++p, ++i) {
    if (p + 1 < p1) fetch(p + 1, nxt, nnxt);
    const int s = i % G.n_stages;
    const uint32_t ph = (uint32_t)(i / G.n_stages) & 1u;
    ok = __all_sync(0xFFFFFFFFu, wait_phase(G.empty + s, ph ^ 1u, G.abort_flag, G.status));
    if (!ok) break;
    fence_proxy_async();
    unsigned char* st = G.stages + (size_t)s * G.stage_bytes;
    if (COPY == 0) {
      int bytes = 0;
#pragma unroll
      for (int k = 0; k < kDescPerLane; ++k)
        if (w + W * (lane + 32 * k) < ncur) bytes += cur[k].w;
      bytes = __reduce_add_sync(0xFFFFFFFFu, bytes);
      if (lane == 0) mbar_expect_tx(G.full + s, (uint32_t)bytes);
      __syncwarp();
#pragma unroll
      for (int k = 0; k < kDescPerLane; ++k)
        if (w + W * (lane + 32 * k) < ncur)
          bulk_load(st + cur[k].z, desc_source(R, tab, cur[k].x, cur[k].y), (uint32_t)cur[k].w, G.full + s);
    } else {
#pragma unroll
      for (int k = 0; k < kDescPerLane; ++k) {
        // this warp's descriptors in slot k sit on lanes 0..nk-1
        const int nk = max(0, min(32, (ncur - w + W - 1) / W - 32 * k));
        for (int j = 0; j < nk; ++j) {
          const int src = __shfl_sync(0xFFFFFFFFu, cur[k].x, j);
          const int row = __shfl_sync(0xFFFFFFFFu, cur[k].y, j);
          const int dst = __shfl_sync(0xFFFFFFFFu, cur[k].z, j);
          const int bytes = __shfl_sync(0xFFFFFFFFu, cur[k].w, j);
          const unsigned char* sp = static_cast<const unsigned char*>(desc_source(R, tab, src, row));
          for (int c = lane * 16; c < bytes; c += 32 * 16) cp16_async(st + dst + c, sp + c);
        }
      }
      cp_async_arrive_noinc(G.full + s);
    }
#pragma unroll
    for (int k = 0; k < kDescPerLane; ++k) cur[k] = nxt[k];
    ncur = nnxt;
  }
  if (!ok) {
    // patches 0..i-1 were issued; wait (bounded) for the copies of the last
    // n_stages of them so none lands after the CTA has exited
    for (int j = max(0, i - G.n_stages); j < i; ++j)
      wait_phase(G.full + j % G.n_stages, (uint32_t)(j / G.n_stages) & 1u, nullptr, G.status);
  }
}

// Compute-warp loop: wait for stage i % n_stages, run `consume` on it, release it.
template <typename Consume>
__device__ __forceinline__ void consume_ring(const Ring& G, int p0, int p1, Consume consume) {
  const int lane = threadIdx.x & 31;
  int i = 0;
  for (int p = p0; p < p1; ++p, ++i) {
    const int s = i % G.n_stages;
    const uint32_t ph = (uint32_t)(i / G.n_stages) & 1u;
    if (!__all_sync(0xFFFFFFFFu, wait_phase(G.full + s, ph, G.abort_flag, G.status))) return;
    consume(G.stages + (size_t)s * G.stage_bytes, s, ph);
    __syncwarp();
    if (lane == 0) mbar_arrive(G.empty + s);
  }
}

// H phase of one patch from its stage (same arithmetic as kh_kernel).
// Surface-impedance poles are handled by groups of T/4 lanes when T/4 is a
// power of two up to 32 (so a group never straddles a warp).
__host__ __device__ inline bool si_lane_groups(int T) {
  const int q = T / 4;
  return T > 0 && (T & 3) == 0 && q <= 32 && (q & (q - 1)) == 0;
}

// Lane layout of the per-run loops.  Thread ct of the nct compute threads
// takes radial quad q = ct % G of the entity rows ct / G, ct / G + per, ...
// (per = nct / G rows per sweep) when q < c, the row's quad count.  G = c
// packs the rows back to back (layout 0); G = c rounded up to a multiple of 8
// (layout 1) starts every row on an 8-lane boundary, so each 8-lane phase of a
// 16-byte shared load reads a single row and gathered rows never meet in one
// phase (no bank conflicts between rows), at the cost of G - c idle lanes per
// row.  Both layouts compute the same values.
struct LaneMap {
  int G, per, q;
  bool on;
};
__device__ __forceinline__ LaneMap lane_map(int ct, int nct, int c, int layout) {
  LaneMap m;
  m.G = layout ? (c + 7) & ~7 : c;
  m.per = nct / m.G;
  m.q = ct % m.G;
  m.on = ct < m.per * m.G && m.q < c;
  return m;
}

template <typename real, bool PLASMA>
__device__ __forceinline__ void kh_consume(const Rec<real>& R, const Layers<real>& Ls, unsigned char* st, int ct,
                                           int nct, uint64_t* group, uint32_t ph, const Ring& G, int layout) {
  constexpr int N = Lanes<real>::N;
  const int* hd = reinterpret_cast<const int*>(st);
  const int ea = hd[kh_ea], ne = hd[kh_ne], fa = hd[kh_fa], nf = hd[kh_nf];
  const real* s_er = reinterpret_cast<const real*>(st + hd[kh_o_er]);
  const real* s_et = reinterpret_cast<const real*>(st + hd[kh_o_et]);
  const real* s_ht = reinterpret_cast<const real*>(st + hd[kh_o_ht]);
  const real* s_hr = reinterpret_cast<const real*>(st + hd[kh_o_hr]);
  const real* s_J = reinterpret_cast<const real*>(st + hd[kh_o_J]);
  const int4* eloc = reinterpret_cast<const int4*>(st + hd[kh_o_eloc]);
  const real* einv = reinterpret_cast<const real*>(st + hd[kh_o_einv]);
  const int4* floc = reinterpret_cast<const int4*>(st + hd[kh_o_floc]);
  const real* fw = reinterpret_cast<const real*>(st + hd[kh_o_fw]);
  const real* fpl = reinterpret_cast<const real*>(st + hd[kh_o_fpl]);
  const real* s_si = reinterpret_cast<const real*>(st + hd[kh_o_si]);
  const real* esis = reinterpret_cast<const real*>(st + hd[kh_o_esis]);
  real* s_hnew = reinterpret_cast<real*>(st + hd[kh_o_hnew]);
  const int T = R.si_terms;
  const bool si_pass = si_lane_groups(T);
  const int Pn = R.Pn, Pm = R.Pm, cn = Pn / N, cm = Pm / N;
  if (si_pass) {
    // each owned edge's surface-impedance ADE on T/4 lanes (four poles each):
    // partial history sums gathered in pole order, the node-0 Ht into the
    // stage's scratch, then all compute warps meet on the slot's group barrier
    const int Q = T / 4, lane = threadIdx.x & 31, n_it = ne * Q;
    for (int base = ct - lane; base < n_it; base += nct) {
      const int it = min(base + lane, n_it - 1);
      const int el = it / Q, qd = it - el * Q;
      const int e = ea + el;
      const int4 loc = eloc[el];
      const real* mem = s_si + el * T;
      const real part = si_quad(mem + 4 * qd, Ls.si_hist + 4 * qd);
      const int first = lane - qd;
      real hist = __shfl_sync(0xFFFFFFFFu, part, first);
      for (int q = 1; q < Q; ++q) hist = add_rn(hist, __shfl_sync(0xFFFFFFFFu, part, first + q));
      const real h_old = s_ht[el * Pn];
      const real g0 = (s_er[loc.y * Pn] - s_er[loc.x * Pn]) * einv[el] * Ls.invr[0];
      const real e1 = R.si_metric * s_et[loc.z * Pm];
      const real h_new = si_boundary(R, h_old, g0, e1, esis[el], hist);
      if (base + lane < n_it) {
        si_update_quad(mem + 4 * qd, R.si_mem + (size_t)e * T + 4 * qd, Ls, 4 * qd, h_new + h_old);
        if (qd == 0) s_hnew[el] = h_new;
      }
    }
    __syncwarp();
    if ((threadIdx.x & 31) == 0) mbar_arrive(group);
    if (!__all_sync(0xFFFFFFFFu, wait_phase(group, ph, G.abort_flag, G.status))) return;
  }
  // edge runs (nodes) and face runs (midpoints), each thread on a fixed
  // radial quad (layer factors loaded once per patch; see ke_consume)
  {
    const LaneMap lm = lane_map(ct, nct, cn, layout);
    if (lm.on) {
      const int k0 = lm.q * N;
      const HEdgeLayer<real> y = h_edge_layer(R, Ls, k0);
      for (int el = ct / lm.G; el < ne; el += lm.per) {
        const int e = ea + el;
        const int4 loc = eloc[el];
        h_edge_run(R, Ls, y, e, k0, s_er + loc.y * Pn, s_er + loc.x * Pn, s_et + loc.z * Pm, s_ht + el * Pn,
                   R.ht + (size_t)e * Pn, einv[el], s_si + el * T, R.si_mem + (size_t)e * T, esis + el,
                   si_pass ? s_hnew + el : nullptr);
      }
    }
  }
  {
    const LaneMap lm = lane_map(ct, nct, cm, layout);
    if (lm.on) {
      const int j0 = lm.q * N;
      const Run<real> fc = ld16(Ls.hC + j0);
      for (int fl = ct / lm.G; fl < nf; fl += lm.per) {
        const int f = fa + fl;
        const int4 l0 = floc[2 * fl];
        const int4 l1 = floc[2 * fl + 1];
        h_face_run<real, PLASMA>(R, Ls, fc, f, j0, s_et + l0.x * Pm, s_et + l0.y * Pm, s_et + l0.z * Pm,
                                 s_hr + fl * Pm, R.hr + (size_t)f * Pm, s_er + l0.w * Pn, s_er + l1.x * Pn,
                                 s_er + l1.y * Pn, s_J + fl * 3 * Pm, nf * 3 * Pm,
                                 R.n_species > 1 ? R.Jtot + (size_t)f * 3 * Pm : nullptr, fw + 4 * fl, fpl + 12 * fl);
      }
    }
  }
}

// E phase of one patch from its stage (same arithmetic as ke_kernel).  Each
// loop gives every thread a fixed radial quad: thread ct takes quad ct % c of
// entities ct / c, ct / c + per, ... (c quads per row, per = nct / c entities
// per sweep; threads from per * c on sit the loop out), so the per-layer
// factors of its quad load once per patch instead of once per run.
template <typename real, bool PLASMA, int MAXDEG>
__device__ __forceinline__ void ke_consume(const Rec<real>& R, const Layers<real>& Ls, unsigned char* st, int ct,
                                           int nct, real current, int layout, unsigned pattern) {
  constexpr int N = Lanes<real>::N;
  const int* hd = reinterpret_cast<const int*>(st);
  const int nv = hd[ke_nv], ea = hd[ke_ea], ne = hd[ke_ne], src = hd[ke_src];
  const real* s_ht = reinterpret_cast<const real*>(st + hd[ke_o_ht]);
  const real* s_hr = reinterpret_cast<const real*>(st + hd[ke_o_hr]);
  const real* s_J = reinterpret_cast<const real*>(st + hd[ke_o_J]);
  const real* s_er = reinterpret_cast<const real*>(st + hd[ke_o_er]);
  const real* s_et = reinterpret_cast<const real*>(st + hd[ke_o_et]);
  const int* vid = reinterpret_cast<const int*>(st + hd[ke_o_vid]);
  const int* vh = reinterpret_cast<const int*>(st + hd[ke_o_vh]);
  const int* vj = reinterpret_cast<const int*>(st + hd[ke_o_vj]);
  const real* vcoef = reinterpret_cast<const real*>(st + hd[ke_o_vcoef]);
  const real* vwc = reinterpret_cast<const real*>(st + hd[ke_o_vwc]);
  const int4* eloc = reinterpret_cast<const int4*>(st + hd[ke_o_eloc]);
  const real* einv = reinterpret_cast<const real*>(st + hd[ke_o_einv]);
  const real* etan = reinterpret_cast<const real*>(st + hd[ke_o_etan]);
  const int Pn = R.Pn, Pm = R.Pm, SW = R.slot_width, cn = Pn / N, cm = Pm / N;
  const bool full = R.coef_full != 0;
  const bool local = PLASMA && R.plasma_local != 0;
  auto slot_rows = [&](int vl, const real** hrows, const real** jrows) {
#pragma unroll
    for (int q = 0; q < MAXDEG; q += 4) {
      const int4 h4 = *reinterpret_cast<const int4*>(vh + vl * SW + q);
      hrows[q] = s_ht + h4.x * Pn;
      hrows[q + 1] = s_ht + h4.y * Pn;
      if (q + 2 < MAXDEG) hrows[q + 2] = s_ht + h4.z * Pn;
      if (q + 3 < MAXDEG) hrows[q + 3] = s_ht + h4.w * Pn;
      if (PLASMA) {
        const int4 j4 = *reinterpret_cast<const int4*>(vj + vl * SW + q);
        jrows[q] = s_J + j4.x * 3 * Pm;
        jrows[q + 1] = s_J + j4.y * 3 * Pm;
        if (q + 2 < MAXDEG) jrows[q + 2] = s_J + j4.z * 3 * Pm;
        if (q + 3 < MAXDEG) jrows[q + 3] = s_J + j4.w * 3 * Pm;
      } else {
        for (int i = 0; i < 4 && q + i < MAXDEG; ++i) jrows[q + i] = nullptr;
      }
    }
  };
  {
    // vertex runs: thread ct holds node quad q of its vertices.  With plasma
    // it computes the vertex's radial current on midpoint quad q itself
    // (midpoints k0 .. k0+N-1) and takes the one below, k0-1, from lane - 1,
    // which holds quad q-1 of the same vertex; a lane whose quad q-1 sits in
    // the previous warp (lane 0) computes that value directly
    const LaneMap lm = lane_map(ct, nct, cn, layout);
    if (lm.on) {
      const int q = lm.q, k0 = q * N, per = lm.per;
      const int lane = threadIdx.x & 31, wbase = ct - lane;
      // the vertex layer factors of this thread's quad: loaded once per patch
      // in the float kernels of vertex degree 6 when they are altitude rows;
      // elsewhere (float64, 12-slot tables) holding them would push the kernel
      // past its register budget into local memory, so they are re-read per run
      constexpr bool kHoist = sizeof(real) == 4 && MAXDEG == 6;
      VertexLayer<real> fixed_v{};
      if (kHoist && !full) fixed_v = vertex_layer(R, Ls, 0, k0);
      for (int k = 0;; ++k) {
        const int vl = ct / lm.G + k * per;
        if (vl >= nv) break;
        // lanes in this iteration: those of the pattern (a valid quad of a
        // row slot) whose thread index is below the sweep's limit
        const int cnt = min(per, nv - k * per) * lm.G - wbase;
        const unsigned mask = pattern & (cnt >= 32 ? 0xFFFFFFFFu : ((1u << cnt) - 1u));
        const int v = vid[vl];
        const real* hrows[MAXDEG];
        const real* jrows[MAXDEG];
        slot_rows(vl, hrows, jrows);
        real rav[N + 1];
        if (PLASMA) {
          const real* wcs = vwc + vl * SW * 4;
          Run<real> own = zero_run<real>();
          if (local) {
            if (k0 < Pm) own = vertex_radial_current_local<real, MAXDEG>(jrows, wcs, k0);
          } else if (k0 < Pm) {
            own = vertex_radial_current<real, MAXDEG>(jrows, wcs, k0, Pm);
          }
          const real below = __shfl_up_sync(mask, own.x[N - 1], 1);
          rav[0] = q == 0   ? real(0)
                   : lane > 0 ? below
                   : local    ? vertex_radial_current_local_at<real, MAXDEG>(jrows, wcs, k0 - 1)
                              : vertex_radial_current_at<real, MAXDEG>(jrows, wcs, k0 - 1, Pm);
#pragma unroll
          for (int r = 0; r < N; ++r) rav[r + 1] = own.x[r];
        }
        e_vertex_run<real, PLASMA, MAXDEG>(R, kHoist && !full ? fixed_v : vertex_layer(R, Ls, v, k0), (src & 1) != 0, v, k0, hrows,
                                           jrows, vcoef + vl * SW, PLASMA ? vwc + vl * SW * 4 : nullptr,
                                           s_er + vl * Pn, R.er + (size_t)v * Pn, current, PLASMA ? rav : nullptr);
      }
    }
  }
  {
    const LaneMap lm = lane_map(ct, nct, cm, layout);
    if (lm.on) {
      const int j0 = lm.q * N;
      const EdgeLayer<real> fixed = edge_layer(R, Ls, ea, j0);
      for (int el = ct / lm.G; el < ne; el += lm.per) {
        const int e = ea + el;
        const int4 loc = eloc[el];
        e_edge_run<real, PLASMA>(R, full ? edge_layer(R, Ls, e, j0) : fixed, (src & 2) != 0, e, j0,
                                 s_hr + loc.y * Pm, s_hr + loc.z * Pm, s_ht + loc.x * Pn,
                                 PLASMA ? s_J + loc.y * 3 * Pm : nullptr, PLASMA ? s_J + loc.z * 3 * Pm : nullptr,
                                 s_et + el * Pm, R.et + (size_t)e * Pm, current, einv[el],
                                 PLASMA ? etan + el * 8 : nullptr);
      }
    }
  }
}

// Bit l set when lane l of this thread's warp holds a valid quad (q < c) in
// the vertex-run lane map: the shuffle mask of the lanes that take part in a
// sweep, before the sweep's row limit is applied.
__device__ __forceinline__ unsigned lane_pattern(int ct, int nct, int c, int layout) {
  const int wbase = ct - (threadIdx.x & 31);
  unsigned bits = 0;
  for (int l = 0; l < 32; ++l)
    if (lane_map(wbase + l, nct, c, layout).on) bits |= 1u << l;
  return bits;
}

// Shared prologue: barriers, record, per-layer rows, this CTA's patch range.
template <typename real>
__device__ __forceinline__ void ring_setup(Rec<real>& R, const Rec<real>* recs, unsigned char* dyn, uint64_t* full,
                                           uint64_t* empty, int* abort_flag, int stage_bytes, int n_stages,
                                           int full_arrivals, int producers, Layers<real>& Ls, Ring& G) {
  if (threadIdx.x == 0) {
    *abort_flag = 0;
    for (int s = 0; s < n_stages; ++s) {
      mbar_init(full + s, full_arrivals);
      mbar_init(empty + s, (blockDim.x - 32 * producers) / 32);
    }
    fence_mbar_init();
  }
  load_rec(R, recs);
  load_layers(R, reinterpret_cast<real*>(dyn), Ls);
  G.stages = dyn + layer_block_bytes(R.layer_reals, (int)sizeof(real));
  G.stage_bytes = stage_bytes;
  G.n_stages = n_stages;
  G.full = full;
  G.empty = empty;
  G.abort_flag = abort_flag;
  G.status = R.status;
}

template <typename real, bool PLASMA, int COPY>
__global__ void __maxnreg__(kMaxRegs) kh_tma(const Rec<real>* __restrict__ recs, int stage_bytes, int n_stages,
                                             int producers, int layout) {
  extern __shared__ __align__(128) unsigned char dyn_smem[];
  __shared__ Rec<real> R;
  __shared__ __align__(8) uint64_t full[kMaxStages], empty[kMaxStages], group[kMaxStages];
  __shared__ int abort_flag;
  Layers<real> Ls;
  Ring G;
  const int W = producers;
  if (threadIdx.x == 0)
    for (int s = 0; s < n_stages; ++s) mbar_init(group + s, (blockDim.x - 32 * W) / 32);  // made visible by ring_setup
  ring_setup(R, recs, dyn_smem, full, empty, &abort_flag, stage_bytes, n_stages, COPY == 0 ? W : 32 * W, W, Ls, G);
  const int n = R.n_patches_h;
  const int p0 = (int)((long long)n * blockIdx.x / gridDim.x), p1 = (int)((long long)n * (blockIdx.x + 1) / gridDim.x);
  if (threadIdx.x < 32 * W) {
    produce<COPY>(R, G, p0, p1, n, R.dptr_h, R.desc_h, R.tab_h, threadIdx.x / 32, W);
  } else {
    const int ct = threadIdx.x - 32 * W, nct = blockDim.x - 32 * W;
    consume_ring(G, p0, p1, [&](unsigned char* st, int s, uint32_t ph) {
      kh_consume<real, PLASMA>(R, Ls, st, ct, nct, group + s, ph, G, layout);
    });
  }
}

template <typename real, bool PLASMA, int MAXDEG, int COPY, int REGS>
__global__ void __maxnreg__(REGS) ke_tma(const Rec<real>* __restrict__ recs, int stage_bytes, int n_stages,
                                         int producers, int istep, int layout) {
  extern __shared__ __align__(128) unsigned char dyn_smem[];
  __shared__ Rec<real> R;
  __shared__ __align__(8) uint64_t full[kMaxStages], empty[kMaxStages];
  __shared__ int abort_flag;
  Layers<real> Ls;
  Ring G;
  const int W = producers;
  ring_setup(R, recs, dyn_smem, full, empty, &abort_flag, stage_bytes, n_stages, COPY == 0 ? W : 32 * W, W, Ls, G);
  const int n = R.n_patches_e;
  const int p0 = (int)((long long)n * blockIdx.x / gridDim.x), p1 = (int)((long long)n * (blockIdx.x + 1) / gridDim.x);
  if (threadIdx.x < 32 * W) {
    produce<COPY>(R, G, p0, p1, n, R.dptr_e, R.desc_e, R.tab_e, threadIdx.x / 32, W);
  } else {
    const int ct = threadIdx.x - 32 * W, nct = blockDim.x - 32 * W;
    const real current = (R.n_src_er + R.n_src_et) > 0 ? (real)R.cur[istep] : real(0);
    const unsigned pattern = lane_pattern(ct, nct, R.Pn / Lanes<real>::N, layout);
    consume_ring(G, p0, p1, [&](unsigned char* st, int s, uint32_t ph) {
      ke_consume<real, PLASMA, MAXDEG>(R, Ls, st, ct, nct, current, layout, pattern);
    });
  }
}

// Batched launches over the members of an ensemble (one launch per phase for
// all members that share the template arguments).  CTA b walks the segments
// segs[sptr[b]] .. segs[sptr[b + 1] - 1], each int4 {member, first patch, end
// patch, 0}, in order; rings[member] = {stage bytes, stages} of that member's
// plan.  Every segment starts from a fresh ring: all threads meet, the
// barriers of the previous segment (all of whose copies have landed and been
// consumed) are invalidated and initialised again, and the member's record
// and per-layer rows are loaded.  The per-patch work is kh_consume /
// ke_consume, so a member's result is the same as its own launch.  A wait that
// runs out ends the CTA's walk after the segment it happened in.
template <typename real>
__device__ __forceinline__ void batch_segment_start(uint64_t* full, uint64_t* empty, uint64_t* group, int prev_stages,
                                                    int n_stages, int compute_warps) {
  if (threadIdx.x == 0) {
    for (int s = 0; s < prev_stages; ++s) {
      mbar_inval(full + s);
      mbar_inval(empty + s);
      mbar_inval(group + s);
    }
    for (int s = 0; s < n_stages; ++s) mbar_init(group + s, compute_warps);  // made visible by ring_setup
  }
}

template <typename real, bool PLASMA, int COPY>
__global__ void __maxnreg__(kMaxRegs) kh_tma_batch(const Rec<real>* __restrict__ recs, const int4* __restrict__ segs,
                                                   const int* __restrict__ sptr, const int2* __restrict__ rings,
                                                   int producers, int layout) {
  extern __shared__ __align__(128) unsigned char dyn_smem[];
  __shared__ Rec<real> R;
  __shared__ __align__(8) uint64_t full[kMaxStages], empty[kMaxStages], group[kMaxStages];
  __shared__ int abort_flag;
  const int W = producers;
  if (threadIdx.x == 0) abort_flag = 0;
  int prev = 0;
  for (int k = sptr[blockIdx.x]; k < sptr[blockIdx.x + 1]; ++k) {
    __syncthreads();
    if (abort_flag) break;
    const int4 sg = segs[k];
    const int2 rg = rings[sg.x];
    batch_segment_start<real>(full, empty, group, prev, rg.y, (blockDim.x - 32 * W) / 32);
    prev = rg.y;
    Layers<real> Ls;
    Ring G;
    ring_setup(R, recs + sg.x, dyn_smem, full, empty, &abort_flag, rg.x, rg.y, COPY == 0 ? W : 32 * W, W, Ls, G);
    if (threadIdx.x < 32 * W) {
      produce<COPY>(R, G, sg.y, sg.z, R.n_patches_h, R.dptr_h, R.desc_h, R.tab_h, threadIdx.x / 32, W);
    } else {
      const int ct = threadIdx.x - 32 * W, nct = blockDim.x - 32 * W;
      consume_ring(G, sg.y, sg.z, [&](unsigned char* st, int s, uint32_t ph) {
        kh_consume<real, PLASMA>(R, Ls, st, ct, nct, group + s, ph, G, layout);
      });
    }
  }
}

template <typename real, bool PLASMA, int MAXDEG, int COPY, int REGS>
__global__ void __maxnreg__(REGS) ke_tma_batch(const Rec<real>* __restrict__ recs, const int4* __restrict__ segs,
                                               const int* __restrict__ sptr, const int2* __restrict__ rings,
                                               int producers, int istep, int layout) {
  extern __shared__ __align__(128) unsigned char dyn_smem[];
  __shared__ Rec<real> R;
  __shared__ __align__(8) uint64_t full[kMaxStages], empty[kMaxStages], group[kMaxStages];
  __shared__ int abort_flag;
  const int W = producers;
  if (threadIdx.x == 0) abort_flag = 0;
  int prev = 0;
  for (int k = sptr[blockIdx.x]; k < sptr[blockIdx.x + 1]; ++k) {
    __syncthreads();
    if (abort_flag) break;
    const int4 sg = segs[k];
    const int2 rg = rings[sg.x];
    batch_segment_start<real>(full, empty, group, prev, rg.y, (blockDim.x - 32 * W) / 32);
    prev = rg.y;
    Layers<real> Ls;
    Ring G;
    ring_setup(R, recs + sg.x, dyn_smem, full, empty, &abort_flag, rg.x, rg.y, COPY == 0 ? W : 32 * W, W, Ls, G);
    if (threadIdx.x < 32 * W) {
      produce<COPY>(R, G, sg.y, sg.z, R.n_patches_e, R.dptr_e, R.desc_e, R.tab_e, threadIdx.x / 32, W);
    } else {
      const int ct = threadIdx.x - 32 * W, nct = blockDim.x - 32 * W;
      const real current = (R.n_src_er + R.n_src_et) > 0 ? (real)R.cur[istep] : real(0);
      const unsigned pattern = lane_pattern(ct, nct, R.Pn / Lanes<real>::N, layout);
      consume_ring(G, sg.y, sg.z, [&](unsigned char* st, int s, uint32_t ph) {
        ke_consume<real, PLASMA, MAXDEG>(R, Ls, st, ct, nct, current, layout, pattern);
      });
    }
  }
}

// Self-test of the bounded wait: one warp waits, with the kernels' own
// wait_phase, for a phase of an mbarrier that nothing arrives on.  The wait
// gives up after kWaitNs, sets bit 0 of *status and the kernel returns; the
// time waited goes to *waited_ns.
__global__ void wait_selftest_kernel(int* status, unsigned long long* waited_ns) {
  __shared__ __align__(8) uint64_t bar;
  __shared__ int abort_flag;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
    abort_flag = 0;
  }
  __syncthreads();
  const uint64_t t0 = global_ns();
  const bool ok = __all_sync(0xFFFFFFFFu, wait_phase(&bar, 0u, &abort_flag, status));
  if (threadIdx.x == 0) *waited_ns = ok ? 0ull : global_ns() - t0;
}

}  // namespace pipe
}  // namespace ifdtd
