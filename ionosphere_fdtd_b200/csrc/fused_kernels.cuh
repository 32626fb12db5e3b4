// Fused leapfrog step: one launch per time step with halo recomputation
// (sm_100a).
//
// The two-launch step (kh then ke, in place) writes the new H to device memory
// and reads it back in the E launch.  Here one CTA per E patch does both
// halves of the step (solver.py:867-869 orders them H then E):
//   1. it computes the new Ht of every edge its E runs read (the edges it owns
//      and the edges incident to the vertices it owns) and the new Hr of every
//      face beside an owned edge, from the old state, into shared memory; the
//      edges and faces it owns also go to the output state;
//   2. after a CTA barrier it computes the new Er of its owned vertices and the
//      new Et of its owned edges from those shared rows and the old E.
// Halo H values are recomputed by every patch that needs them, with the same
// arithmetic as their owner (the run functions of step_kernels.cuh), so the
// results equal the two-launch step bit for bit.  Neighbouring patches read
// the old E and H while the owners write the new ones, so the step reads one
// state (rin) and writes another (rout): the plan keeps a second copy of the
// four field arrays and alternates between them.  Plasma and the surface
// impedance ADE are not fused (their state would need the same double buffer,
// and the plasma current's halo widens to every face around an owned vertex).
//
// Two kernels: fused_step_kernel gathers straight from global memory (one CTA
// per patch); pipe::kf_tma stages each patch's old rows through the
// warp-specialised ring of pipe_kernels.cuh and updates H in place in the
// stage.
#pragma once

#include "pipe_kernels.cuh"
#include "step_kernels.cuh"

namespace ifdtd {

// Per-patch tables of the fused step (device pointers).  Patch p's halo edge
// list is hedge[patch[p].x .. patch[p+1].x), its first patch[p].y entries
// being the edges it owns (eptr_e order); its face list is
// hface[patch[p].z .. patch[p+1].z), the first patch[p].w being the faces it
// writes.  vslot[slot * slot_width + q] is the position in the patch's edge
// list of vertex slot q's edge; eface[e] the positions in the face list of
// owned edge e's left and right faces.
struct FusedTables {
  const int4* patch;
  const int* hedge;
  const int* hface;
  const int* vslot;
  const int2* eface;
};

template <typename real>
__device__ __forceinline__ void st_shared16(real* p, const Run<real>& r) {
  if constexpr (sizeof(real) == 4) {
    *reinterpret_cast<float4*>(p) = make_float4(r.x[0], r.x[1], r.x[2], r.x[3]);
  } else {
    *reinterpret_cast<double2*>(p) = make_double2(r.x[0], r.x[1]);
  }
}

template <typename real, int MAXDEG>
__global__ void __launch_bounds__(256) fused_step_kernel(const Rec<real>* __restrict__ rin,
                                                         const Rec<real>* __restrict__ rout, FusedTables ft, int istep) {
  constexpr int N = Lanes<real>::N;
  extern __shared__ __align__(16) unsigned char dyn_smem[];
  __shared__ Rec<real> R;
  const int patch = blockIdx.x;
  load_rec(R, rin);
  Layers<real> Ls;
  load_layers(R, reinterpret_cast<real*>(dyn_smem), Ls);
  real* const er_out = rout->er;
  real* const et_out = rout->et;
  real* const hr_out = rout->hr;
  real* const ht_out = rout->ht;
  const int Pn = R.Pn, Pm = R.Pm, SW = R.slot_width, cn = Pn / N, cm = Pm / N;
  const uint32_t mag_cn = div_magic(cn), mag_cm = div_magic(cm);
  const int4 p0 = __ldg(ft.patch + patch), p1 = __ldg(ft.patch + patch + 1);
  const int nhe = p1.x - p0.x, own_e = p0.y, nhf = p1.z - p0.z, own_f = p0.w;
  // the new H rows of the patch's halo, after the per-layer rows (16-byte aligned)
  real* const s_ht = reinterpret_cast<real*>(dyn_smem) + (R.layer_reals + 3) / 4 * 4;
  real* const s_hr = s_ht + (size_t)nhe * Pn;
  // 1. new Ht (edges) and Hr (faces) from the old state
  for (int it = threadIdx.x; it < nhe * cn; it += blockDim.x) {
    const int el = fast_div(it, mag_cn);
    const int e = __ldg(ft.hedge + p0.x + el);
    const int2 th = __ldg(R.edge_th + e);
    const int k0 = (it - el * cn) * N;
    const Run<real> v = h_edge_value(R, Ls, h_edge_layer(R, Ls, k0), e, k0, R.er + (size_t)th.y * Pn,
                                     R.er + (size_t)th.x * Pn, R.et + (size_t)e * Pm, R.ht + (size_t)e * Pn,
                                     __ldg(R.inv_theta + e), (const real*)nullptr, (real*)nullptr,
                                     (const real*)nullptr, (const real*)nullptr);
    st_shared16(s_ht + el * Pn + k0, v);
    if (el < own_e) st16(ht_out + (size_t)e * Pn + k0, v);
  }
  for (int it = threadIdx.x; it < nhf * cm; it += blockDim.x) {
    const int fl = fast_div(it, mag_cm);
    const int f = __ldg(ft.hface + p0.z + fl);
    const int4 fe = __ldg(R.face_e + f);
    const int j0 = (it - fl * cm) * N;
    real wv[4];
    ld4(R.face_w + 4 * (size_t)f, wv);
    const Run<real> v = hr_value(ld16(R.hr + (size_t)f * Pm + j0), ld16(R.et + (size_t)fe.x * Pm + j0),
                                 ld16(R.et + (size_t)fe.y * Pm + j0), ld16(R.et + (size_t)fe.z * Pm + j0), wv[0], wv[1],
                                 wv[2], ld16(Ls.hC + j0));
    st_shared16(s_hr + fl * Pm + j0, v);
    if (fl < own_f) st16(hr_out + (size_t)f * Pm + j0, v);
  }
  __syncthreads();
  // 2. new Er (owned vertices) and Et (owned edges) from the shared H rows
  const real current = (R.n_src_er + R.n_src_et) > 0 ? (real)R.cur[istep] : real(0);
  const int va = R.vptr[patch], vb = R.vptr[patch + 1];
  for (int it = threadIdx.x; it < (vb - va) * cn; it += blockDim.x) {
    const int vl = fast_div(it, mag_cn);
    const int slot = va + vl;
    const int v = __ldg(R.vlist + slot);
    const real* hrows[MAXDEG];
    const real* jrows[MAXDEG];
#pragma unroll
    for (int q = 0; q < MAXDEG; ++q) {
      hrows[q] = s_ht + __ldg(ft.vslot + (size_t)slot * SW + q) * Pn;
      jrows[q] = nullptr;
    }
    const int k0 = (it - vl * cn) * N;
    e_vertex_run<real, false, MAXDEG>(R, vertex_layer(R, Ls, v, k0), R.n_src_er > 0, v, k0, hrows, jrows,
                                      R.ps_coef + (size_t)slot * SW, nullptr, R.er + (size_t)v * Pn,
                                      er_out + (size_t)v * Pn, current);
  }
  const int ea = R.eptr_e[patch], eb = R.eptr_e[patch + 1];
  for (int it = threadIdx.x; it < (eb - ea) * cm; it += blockDim.x) {
    const int el = fast_div(it, mag_cm);
    const int e = ea + el;
    const int2 lf = __ldg(ft.eface + e);
    const int j0 = (it - el * cm) * N;
    e_edge_run<real, false>(R, edge_layer(R, Ls, e, j0), R.n_src_et > 0, e, j0, s_hr + (size_t)lf.x * Pm,
                            s_hr + (size_t)lf.y * Pm, s_ht + (size_t)el * Pn, nullptr, nullptr, R.et + (size_t)e * Pm,
                            et_out + (size_t)e * Pm, current, __ldg(R.inv_phi + e), nullptr);
  }
}

namespace pipe {

// Fused-step blob header (ints; offsets are bytes from the stage start).  The
// stage holds the old er rows of every vertex an H edge touches (the owned
// vertices among them), the old et rows of the H edges and of the edges of
// the H faces, and the old ht / hr rows of the H edges / faces, which the
// consumer overwrites in place with the new values.
enum KfHead : int {
  kf_nhe, kf_nhf, kf_nv, kf_ea, kf_ne, kf_o_er, kf_o_et, kf_o_ht, kf_o_hr,
  kf_o_hel, kf_o_hinv, kf_o_hid, kf_o_fel, kf_o_fw, kf_o_fid,
  kf_o_vid, kf_o_vh, kf_o_vcoef, kf_o_vel, kf_o_eloc, kf_o_einv, kf_src, kf_o_end, kf_head_ints = 24
};
// hel[i]: stage rows of H edge i's head er, tail er, et and ht; hid[i]: its
// edge id, bit 31 set when another patch owns it (computed, not written);
// fel[i]: stage rows of H face i's three edges' et and its hr; fid[i] as hid.
// vh: ht stage rows of the owned vertices' slots; vel: their er stage rows;
// eloc[el]: stage rows of owned edge el's ht, left hr, right hr and et.
constexpr int kNotOwned = (int)0x80000000u;

template <typename real, int MAXDEG>
__device__ __forceinline__ void kf_consume(const Rec<real>& R, const Layers<real>& Ls, unsigned char* st, int ct,
                                           int nct, real current, int layout, uint64_t* group, uint32_t ph,
                                           const Ring& G, real* er_out, real* et_out, real* hr_out, real* ht_out) {
  constexpr int N = Lanes<real>::N;
  const int* hd = reinterpret_cast<const int*>(st);
  const int nhe = hd[kf_nhe], nhf = hd[kf_nhf], nv = hd[kf_nv], ea = hd[kf_ea], ne = hd[kf_ne], src = hd[kf_src];
  const real* s_er = reinterpret_cast<const real*>(st + hd[kf_o_er]);
  const real* s_et = reinterpret_cast<const real*>(st + hd[kf_o_et]);
  real* s_ht = reinterpret_cast<real*>(st + hd[kf_o_ht]);
  real* s_hr = reinterpret_cast<real*>(st + hd[kf_o_hr]);
  const int4* hel = reinterpret_cast<const int4*>(st + hd[kf_o_hel]);
  const real* hinv = reinterpret_cast<const real*>(st + hd[kf_o_hinv]);
  const int* hid = reinterpret_cast<const int*>(st + hd[kf_o_hid]);
  const int4* fel = reinterpret_cast<const int4*>(st + hd[kf_o_fel]);
  const real* fw = reinterpret_cast<const real*>(st + hd[kf_o_fw]);
  const int* fid = reinterpret_cast<const int*>(st + hd[kf_o_fid]);
  const int* vid = reinterpret_cast<const int*>(st + hd[kf_o_vid]);
  const int* vh = reinterpret_cast<const int*>(st + hd[kf_o_vh]);
  const real* vcoef = reinterpret_cast<const real*>(st + hd[kf_o_vcoef]);
  const int* vel = reinterpret_cast<const int*>(st + hd[kf_o_vel]);
  const int4* eloc = reinterpret_cast<const int4*>(st + hd[kf_o_eloc]);
  const real* einv = reinterpret_cast<const real*>(st + hd[kf_o_einv]);
  const int Pn = R.Pn, Pm = R.Pm, SW = R.slot_width, cn = Pn / N, cm = Pm / N;
  // 1. new Ht and Hr of the patch's H edges and faces, in place (each thread
  // reads and writes only its own quad of a row)
  {
    const LaneMap lm = lane_map(ct, nct, cn, layout);
    if (lm.on) {
      const int k0 = lm.q * N;
      const HEdgeLayer<real> y = h_edge_layer(R, Ls, k0);
      for (int i = ct / lm.G; i < nhe; i += lm.per) {
        const int4 l = hel[i];
        const int raw = hid[i], e = raw & 0x7FFFFFFF;
        const Run<real> v = h_edge_value(R, Ls, y, e, k0, s_er + l.x * Pn, s_er + l.y * Pn, s_et + l.z * Pm,
                                         s_ht + l.w * Pn, hinv[i], (const real*)nullptr, (real*)nullptr,
                                         (const real*)nullptr, (const real*)nullptr);
        st_shared16(s_ht + l.w * Pn + k0, v);
        if (raw >= 0) st16(ht_out + (size_t)e * Pn + k0, v);
      }
    }
  }
  {
    const LaneMap lm = lane_map(ct, nct, cm, layout);
    if (lm.on) {
      const int j0 = lm.q * N;
      const Run<real> fc = ld16(Ls.hC + j0);
      for (int i = ct / lm.G; i < nhf; i += lm.per) {
        const int4 l = fel[i];
        const int raw = fid[i], f = raw & 0x7FFFFFFF;
        real w[4];
        ld4(fw + 4 * i, w);
        const Run<real> v = hr_value(ld16(s_hr + l.w * Pm + j0), ld16(s_et + l.x * Pm + j0), ld16(s_et + l.y * Pm + j0),
                                     ld16(s_et + l.z * Pm + j0), w[0], w[1], w[2], fc);
        st_shared16(s_hr + l.w * Pm + j0, v);
        if (raw >= 0) st16(hr_out + (size_t)f * Pm + j0, v);
      }
    }
  }
  // every compute warp's new H rows are in place before any E run reads them
  __syncwarp();
  if ((threadIdx.x & 31) == 0) mbar_arrive(group);
  if (!__all_sync(0xFFFFFFFFu, wait_phase(group, ph, G.abort_flag, G.status))) return;
  // 2. new Er (owned vertices) and Et (owned edges)
  {
    const LaneMap lm = lane_map(ct, nct, cn, layout);
    if (lm.on) {
      const int k0 = lm.q * N;
      for (int vl = ct / lm.G; vl < nv; vl += lm.per) {
        const int v = vid[vl];
        const real* hrows[MAXDEG];
        const real* jrows[MAXDEG];
#pragma unroll
        for (int q = 0; q < MAXDEG; q += 4) {
          const int4 h4 = *reinterpret_cast<const int4*>(vh + vl * SW + q);
          hrows[q] = s_ht + h4.x * Pn;
          hrows[q + 1] = s_ht + h4.y * Pn;
          if (q + 2 < MAXDEG) hrows[q + 2] = s_ht + h4.z * Pn;
          if (q + 3 < MAXDEG) hrows[q + 3] = s_ht + h4.w * Pn;
        }
#pragma unroll
        for (int q = 0; q < MAXDEG; ++q) jrows[q] = nullptr;
        e_vertex_run<real, false, MAXDEG>(R, vertex_layer(R, Ls, v, k0), (src & 1) != 0, v, k0, hrows, jrows,
                                          vcoef + vl * SW, nullptr, s_er + vel[vl] * Pn, er_out + (size_t)v * Pn,
                                          current);
      }
    }
  }
  {
    const LaneMap lm = lane_map(ct, nct, cm, layout);
    if (lm.on) {
      const int j0 = lm.q * N;
      const bool full = R.coef_full != 0;
      const EdgeLayer<real> fixed = edge_layer(R, Ls, ea, j0);
      for (int el = ct / lm.G; el < ne; el += lm.per) {
        const int e = ea + el;
        const int4 l = eloc[el];
        e_edge_run<real, false>(R, full ? edge_layer(R, Ls, e, j0) : fixed, (src & 2) != 0, e, j0, s_hr + l.y * Pm,
                                s_hr + l.z * Pm, s_ht + l.x * Pn, nullptr, nullptr, s_et + l.w * Pm,
                                et_out + (size_t)e * Pm, current, einv[el], nullptr);
      }
    }
  }
}

// Fused step through the ring: the patches are the E-phase patches (their
// copy descriptors and blobs in the record's E-phase table fields); rin holds
// the old state the copies read, rout the arrays the new state goes to.
template <typename real, int MAXDEG, int COPY>
__global__ void __maxnreg__(kMaxRegs) kf_tma(const Rec<real>* __restrict__ rin, const Rec<real>* __restrict__ rout,
                                             int stage_bytes, int n_stages, int producers, int istep, int layout) {
  extern __shared__ __align__(128) unsigned char dyn_smem[];
  __shared__ Rec<real> R;
  __shared__ __align__(8) uint64_t full[kMaxStages], empty[kMaxStages], group[kMaxStages];
  __shared__ int abort_flag;
  Layers<real> Ls;
  Ring G;
  const int W = producers;
  if (threadIdx.x == 0)
    for (int s = 0; s < n_stages; ++s) mbar_init(group + s, (blockDim.x - 32 * W) / 32);  // made visible by ring_setup
  ring_setup(R, rin, dyn_smem, full, empty, &abort_flag, stage_bytes, n_stages, COPY == 0 ? W : 32 * W, W, Ls, G);
  const int n = R.n_patches_e;
  const int p0 = (int)((long long)n * blockIdx.x / gridDim.x), p1 = (int)((long long)n * (blockIdx.x + 1) / gridDim.x);
  if (threadIdx.x < 32 * W) {
    produce<COPY>(R, G, p0, p1, n, R.dptr_e, R.desc_e, R.tab_e, threadIdx.x / 32, W);
  } else {
    real* const er_out = rout->er;
    real* const et_out = rout->et;
    real* const hr_out = rout->hr;
    real* const ht_out = rout->ht;
    const int ct = threadIdx.x - 32 * W, nct = blockDim.x - 32 * W;
    const real current = (R.n_src_er + R.n_src_et) > 0 ? (real)R.cur[istep] : real(0);
    consume_ring(G, p0, p1, [&](unsigned char* st, int s, uint32_t ph) {
      kf_consume<real, MAXDEG>(R, Ls, st, ct, nct, current, layout, group + s, ph, G, er_out, et_out, hr_out, ht_out);
    });
  }
}

// Batched fused step over ensemble members that share the template
// arguments (the walk of kh_tma_batch): CTA b walks segments
// segs[sptr[b]] .. segs[sptr[b + 1] - 1] = {member, first patch, end patch, 0};
// rin[member] / rout[member] are that member's records of the copy it reads
// and the copy it writes; rings[member] = {stage bytes, stages}.
template <typename real, int MAXDEG, int COPY>
__global__ void __maxnreg__(kMaxRegs) kf_tma_batch(const Rec<real>* __restrict__ rin, const Rec<real>* __restrict__ rout,
                                                   const int4* __restrict__ segs, const int* __restrict__ sptr,
                                                   const int2* __restrict__ rings, int producers, int istep,
                                                   int layout) {
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
    ring_setup(R, rin + sg.x, dyn_smem, full, empty, &abort_flag, rg.x, rg.y, COPY == 0 ? W : 32 * W, W, Ls, G);
    if (threadIdx.x < 32 * W) {
      produce<COPY>(R, G, sg.y, sg.z, R.n_patches_e, R.dptr_e, R.desc_e, R.tab_e, threadIdx.x / 32, W);
    } else {
      const Rec<real>* ro = rout + sg.x;
      real* const er_out = ro->er;
      real* const et_out = ro->et;
      real* const hr_out = ro->hr;
      real* const ht_out = ro->ht;
      const int ct = threadIdx.x - 32 * W, nct = blockDim.x - 32 * W;
      const real current = (R.n_src_er + R.n_src_et) > 0 ? (real)R.cur[istep] : real(0);
      consume_ring(G, sg.y, sg.z, [&](unsigned char* st, int s, uint32_t ph) {
        kf_consume<real, MAXDEG>(R, Ls, st, ct, nct, current, layout, group + s, ph, G, er_out, et_out, hr_out, ht_out);
      });
    }
  }
}

}  // namespace pipe
}  // namespace ifdtd
