// Device kernels of the geodesic FDTD time step (sm_100a).
//
// One launch record (Rec) describes one simulation: its device tables, its
// state pointers and the per-layer radial metric.  A CTA owns a "patch": a
// contiguous range of faces [f0, f0+fpp), the edges first met while scanning
// those faces (a contiguous edge range, because the reference numbers edges in
// face-scan order, mesh.py:674-708) and the vertices whose lowest-numbered
// incident face lies in the range (listed in vlist).
//
// Work mapping: a thread owns a run of RUN consecutive radial samples of one
// column (a "chunk").  Per-column indices and metric factors are loaded once
// per chunk and the RUN samples of every gathered neighbour column are
// independent loads, so each thread keeps many loads in flight; a warp covers
// 32 chunks, i.e. a few columns of consecutive memory.  Vertex gathers use
// fixed-width slot tables (MAXDEG slots, padded with coefficient 0 exactly as
// the reference pads its incidence table, torch_backend.py:66-89), stored in
// patch order so the index chain is two loads deep and the loops unroll.
// Per-layer metric factors and altitude-only coefficient rows are staged in
// shared memory.
//
// Two in-place launches form one leapfrog step, in the reference's order
// (solver.py:867-989):
//   kh_kernel: Ht (edges, nodes 0..L) with the lower surface-impedance ADE,
//              Hr (faces, midpoints) and the cold-plasma current ADE (faces).
//   ke_kernel: Er (vertices, nodes) and Et (edges, midpoints) with the
//              loss integrator, source injection and plasma current coupling.
// kh writes only H and plasma state and reads E; ke writes only E and reads H
// and the new plasma state, so both are race-free in place.  All sums run in a
// fixed order: results are bitwise repeatable and independent of the patch
// size.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace ifdtd {

constexpr int kMaxSpecies = 4;

template <typename real>
struct Rec {
  // sizes and switches
  int nV, nE, nF, L;
  int n_patches, fpp;
  int full, si_terms, n_species, plasma_full, magnetized, coef_full;
  int n_src_er, n_src_et;
  int src_er_vmin, src_er_vmax, src_et_emin, src_et_emax;
  int maxdeg, layer_reals;
  // state
  real *er, *et, *hr, *ht, *si_mem;
  real* J[kMaxSpecies];
  real* Jtot;            // summed species current when n_species > 1
  const double* cur;     // per-step source current (staging row)
  // patch ownership
  const int *eptr, *vptr, *vlist;
  // edges
  const int2 *edge_th, *edge_lr;
  const real *inv_theta, *inv_phi;
  // faces
  const int4 *face_e, *face_v;
  const real* face_w;    // (F,3): sign_i * theta_i / A_f
  // vertex slots in vlist order: (V, maxdeg) edges / coefficients / faces / weighted centres
  const int* ps_edge;
  const real* ps_coef;   // sign * phi_e / A*_v, 0 in padding slots
  const int* ps_face;
  const real* ps_wc;     // (V, maxdeg, 3): area weight * face centre, 0 in padding slots
  // radial metric (global copies; kernels stage them in shared memory)
  const real *invr, *rr, *mid, *invm, *invdr, *invcd;
  real dtmu;             // dt / mu0
  // loss coefficients: (rows, L+1) / (rows, L), rows = 1 or V / E
  const real *ca_er, *cb_er, *ca_et, *cb_et;
  // sources
  const int *src_er_v, *src_er_k;
  const real* src_er_c;
  const int *src_et_e, *src_et_j;
  const real* src_et_c;
  // surface impedance
  real si_metric, si_kappa, si_hist_sum;
  const real *si_scale, *si_decay, *si_drive, *si_hist;
  // plasma
  const real *recon, *centre, *tan_l, *tan_r;
  const real *pcoef, *bdir;
};

// Shared-memory view of the per-layer rows of one record.
template <typename real>
struct Layers {
  real *invr, *rr, *invcd, *mid, *invm, *invdr;
  real *ca_er, *cb_er, *ca_et, *cb_et;  // compressed coefficient rows (else null)
  real *pc, *bd;                        // compressed plasma rows (else null)
};

// Number of reals of per-layer data staged in shared memory (host and device).
__host__ __device__ inline int layer_reals(int L, int coef_full, int species, int plasma_full, int magnetized) {
  int n = 3 * (L + 1) + 3 * L;
  if (!coef_full) n += 2 * (L + 1) + 2 * L;
  if (species > 0 && !plasma_full) n += 6 * species * L + (magnetized ? 3 * L : 0);
  return n;
}

// Copy the launch record into shared memory (one coalesced read per CTA).
template <typename real>
__device__ __forceinline__ void load_rec(Rec<real>& dst, const Rec<real>* src) {
  static_assert(sizeof(Rec<real>) % 4 == 0, "record must be word sized");
  const int words = sizeof(Rec<real>) / 4;
  const uint32_t* s = reinterpret_cast<const uint32_t*>(src);
  uint32_t* d = reinterpret_cast<uint32_t*>(&dst);
  for (int i = threadIdx.x; i < words; i += blockDim.x) d[i] = __ldg(s + i);
  __syncthreads();
}

template <typename real>
__device__ __forceinline__ void copy_row(real* dst, const real* src, int n) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = __ldg(src + i);
}

// Carve and fill the shared per-layer rows; ends with a barrier.
template <typename real>
__device__ __forceinline__ void load_layers(const Rec<real>& R, real* smem, Layers<real>& Ls) {
  const int L = R.L, Lp1 = L + 1;
  real* p = smem;
  Ls.invr = p; p += Lp1;
  Ls.rr = p; p += Lp1;
  Ls.invcd = p; p += Lp1;
  Ls.mid = p; p += L;
  Ls.invm = p; p += L;
  Ls.invdr = p; p += L;
  copy_row(Ls.invr, R.invr, Lp1);
  copy_row(Ls.rr, R.rr, Lp1);
  copy_row(Ls.invcd, R.invcd, Lp1);
  copy_row(Ls.mid, R.mid, L);
  copy_row(Ls.invm, R.invm, L);
  copy_row(Ls.invdr, R.invdr, L);
  Ls.ca_er = Ls.cb_er = Ls.ca_et = Ls.cb_et = nullptr;
  if (!R.coef_full) {
    Ls.ca_er = p; p += Lp1;
    Ls.cb_er = p; p += Lp1;
    Ls.ca_et = p; p += L;
    Ls.cb_et = p; p += L;
    copy_row(Ls.ca_er, R.ca_er, Lp1);
    copy_row(Ls.cb_er, R.cb_er, Lp1);
    copy_row(Ls.ca_et, R.ca_et, L);
    copy_row(Ls.cb_et, R.cb_et, L);
  }
  Ls.pc = Ls.bd = nullptr;
  if (R.n_species > 0 && !R.plasma_full) {
    Ls.pc = p; p += 6 * R.n_species * L;
    copy_row(Ls.pc, R.pcoef, 6 * R.n_species * L);
    if (R.magnetized) {
      Ls.bd = p; p += 3 * L;
      copy_row(Ls.bd, R.bdir, 3 * L);
    }
  }
  __syncthreads();
}

// q = n / d for n < 2^24 and 1 <= d <= 1024 with m = ceil(2^32 / d); d = 1
// (m = 2^32 does not fit) is encoded as m = 0 and divides as the identity.
__device__ __forceinline__ int fast_div(int n, uint32_t m) { return m ? (int)__umulhi((uint32_t)n, m) : n; }
__device__ __forceinline__ uint32_t div_magic(int d) { return d == 1 ? 0u : 0xFFFFFFFFu / (uint32_t)d + 1u; }

template <typename real>
__device__ __forceinline__ real pcoef_at(const Rec<real>& R, const Layers<real>& Ls, int s, int c, int f, int j) {
  if (!R.plasma_full) return Ls.pc[(s * 6 + c) * R.L + j];
  return __ldg(R.pcoef + (((size_t)(s * 6 + c) * R.nF + f) * R.L + j));
}

template <typename real>
__device__ __forceinline__ const real* jsum(const Rec<real>& R) {
  return R.n_species > 1 ? R.Jtot : R.J[0];
}

__device__ __forceinline__ void member_patch(const int2* block_map, int n_members, int& member, int& patch) {
  member = 0;
  patch = blockIdx.x;
  if (n_members > 1) {
    const int2 bm = block_map[blockIdx.x];
    member = bm.x;
    patch = bm.y;
  }
}

// ---------------------------------------------------------------------------
// H phase: Ht (edges x nodes), surface-impedance ADE, Hr (faces x midpoints),
// cold-plasma current ADE (faces x midpoints).
// solver.py:877-921; surface_impedance.py:225-270; plasma.py:413-442, 489-501.
// ---------------------------------------------------------------------------
template <typename real, bool PLASMA, int RUN>
__global__ void __launch_bounds__(256) kh_kernel(const Rec<real>* __restrict__ recs, const int2* __restrict__ block_map,
                                                  int n_members) {
  extern __shared__ __align__(16) unsigned char dyn_smem[];
  __shared__ Rec<real> R;
  int member, patch;
  member_patch(block_map, n_members, member, patch);
  load_rec(R, recs + member);
  Layers<real> Ls;
  load_layers(R, reinterpret_cast<real*>(dyn_smem), Ls);
  const int L = R.L, Lp1 = L + 1;
  const int cn = (Lp1 + RUN - 1) / RUN, cm = (L + RUN - 1) / RUN;
  const uint32_t mag_cn = div_magic(cn), mag_cm = div_magic(cm);
  const real* __restrict__ er = R.er;
  const real* __restrict__ et = R.et;
  real* __restrict__ ht = R.ht;
  real* __restrict__ hr = R.hr;
  const real dtmu = R.dtmu;
  const bool si = R.si_terms > 0;
  const bool full = R.full != 0;

  // ---- Ht: d/dt Ht = (grad_s Er - (1/r) d(m Et)/dr) / mu0, odd (PEC) Et ghosts ----
  const int ea = R.eptr[patch], eb = R.eptr[patch + 1];
  const int n_edge_items = (eb - ea) * cn;
  for (int it = threadIdx.x; it < n_edge_items; it += blockDim.x) {
    const int el = fast_div(it, mag_cn);
    const int k0 = (it - el * cn) * RUN;
    const int e = ea + el;
    const int2 th = __ldg(R.edge_th + e);
    const real inv_t = __ldg(R.inv_theta + e);
    const real* erh = er + (size_t)th.y * Lp1;
    const real* ert = er + (size_t)th.x * Lp1;
    const real* etr = et + (size_t)e * L;
    real* htr = ht + (size_t)e * Lp1;
    real vh[RUN], vt[RUN], vo[RUN], vu[RUN + 1];
#pragma unroll
    for (int r = 0; r < RUN; ++r) {
      const int k = k0 + r;
      const bool ok = k < Lp1;
      vh[r] = ok ? erh[k] : real(0);
      vt[r] = ok ? ert[k] : real(0);
      vo[r] = ok ? htr[k] : real(0);
    }
#pragma unroll
    for (int r = 0; r <= RUN; ++r) {
      const int k = k0 - 1 + r;
      vu[r] = (k >= 0 && k < L) ? etr[k] : real(0);
    }
#pragma unroll
    for (int r = 0; r < RUN; ++r) {
      const int k = k0 + r;
      if (k >= Lp1 || (si && k == 0)) continue;  // the surface ADE owns the lowest plane
      const real g = (vh[r] - vt[r]) * inv_t * Ls.invr[k];
      real up = vu[r + 1], dn = vu[r];
      real d;
      if (full) {
        up = (k < L) ? up * Ls.mid[k] : real(0);
        dn = (k > 0) ? dn * Ls.mid[k - 1] : real(0);
        d = (up - dn) * Ls.invcd[k] * Ls.invr[k];
      } else {
        d = (up - dn) * Ls.invcd[k];
      }
      htr[k] = vo[r] + (g - d) * dtmu;
    }
  }

  // ---- lower surface-impedance boundary (implicit, trapezoidal ADE) ----
  if (si) {
    const int T = R.si_terms;
    for (int el = threadIdx.x; el < eb - ea; el += blockDim.x) {
      const int e = ea + el;
      const int2 th = __ldg(R.edge_th + e);
      const real h_old = ht[(size_t)e * Lp1];
      const real g0 = (er[(size_t)th.y * Lp1] - er[(size_t)th.x * Lp1]) * __ldg(R.inv_theta + e) * Ls.invr[0];
      const real e1 = R.si_metric * et[(size_t)e * L];
      const real s = __ldg(R.si_scale + e);
      real* mem = R.si_mem + (size_t)e * T;
      real hist = real(0);
      for (int p = 0; p < T; ++p) hist += mem[p] * __ldg(R.si_hist + p);
      hist *= s;
      const real kap = R.si_kappa;
      const real c = kap * (s * R.si_hist_sum);
      const real h_new = ((real(1) - real(0.5) * c) * h_old + dtmu * g0 - kap * e1 + kap * hist) / (real(1) + real(0.5) * c);
      ht[(size_t)e * Lp1] = h_new;
      const real hs = h_new + h_old;
      for (int p = 0; p < T; ++p) mem[p] = mem[p] * __ldg(R.si_decay + p) + hs * __ldg(R.si_drive + p);
    }
  }

  // ---- Hr and the plasma current on owned faces ----
  const int fa = patch * R.fpp;
  const int fb = min(fa + R.fpp, R.nF);
  const int n_face_items = (fb - fa) * cm;
  for (int it = threadIdx.x; it < n_face_items; it += blockDim.x) {
    const int fl = fast_div(it, mag_cm);
    const int j0 = (it - fl * cm) * RUN;
    const int f = fa + fl;
    const int4 fe = __ldg(R.face_e + f);
    const real w0 = __ldg(R.face_w + 3 * (size_t)f), w1 = __ldg(R.face_w + 3 * (size_t)f + 1),
               w2 = __ldg(R.face_w + 3 * (size_t)f + 2);
    const real* et0 = et + (size_t)fe.x * L;
    const real* et1 = et + (size_t)fe.y * L;
    const real* et2 = et + (size_t)fe.z * L;
    real* hrr = hr + (size_t)f * L;
    real a0[RUN], a1[RUN], a2[RUN], hv[RUN];
#pragma unroll
    for (int r = 0; r < RUN; ++r) {
      const int j = j0 + r;
      const bool ok = j < L;
      a0[r] = ok ? et0[j] : real(0);
      a1[r] = ok ? et1[j] : real(0);
      a2[r] = ok ? et2[j] : real(0);
      hv[r] = ok ? hrr[j] : real(0);
    }
#pragma unroll
    for (int r = 0; r < RUN; ++r) {
      const int j = j0 + r;
      if (j < L) hrr[j] = hv[r] - (w0 * a0[r] + w1 * a1[r] + w2 * a2[r]) * Ls.invm[j] * dtmu;
    }
    if (PLASMA) {
      const int4 fv = __ldg(R.face_v + f);
      const real* va = er + (size_t)fv.x * Lp1;
      const real* vb = er + (size_t)fv.y * Lp1;
      const real* vc = er + (size_t)fv.z * Lp1;
      real node[RUN + 1];
      const real third = real(1) / real(3);
#pragma unroll
      for (int r = 0; r <= RUN; ++r) {
        const int k = j0 + r;
        node[r] = (k <= L) ? (va[k] + vb[k] + vc[k]) * third : real(0);
      }
      real rc[9], cf[3];
#pragma unroll
      for (int c = 0; c < 9; ++c) rc[c] = __ldg(R.recon + 9 * (size_t)f + c);
#pragma unroll
      for (int c = 0; c < 3; ++c) cf[c] = __ldg(R.centre + 3 * (size_t)f + c);
      real E[RUN][3];
#pragma unroll
      for (int r = 0; r < RUN; ++r) {
        const real rad = real(0.5) * (node[r] + node[r + 1]);
#pragma unroll
        for (int c = 0; c < 3; ++c) E[r][c] = a0[r] * rc[c] + a1[r] * rc[3 + c] + a2[r] * rc[6 + c] + rad * cf[c];
      }
      real tot[RUN][3];
#pragma unroll
      for (int r = 0; r < RUN; ++r) tot[r][0] = tot[r][1] = tot[r][2] = real(0);
      for (int s = 0; s < R.n_species; ++s) {
        real* Js = R.J[s] + ((size_t)f * L) * 3;
        real jv[RUN][3];
#pragma unroll
        for (int r = 0; r < RUN; ++r) {
          const int j = j0 + r;
#pragma unroll
          for (int c = 0; c < 3; ++c) jv[r][c] = (j < L) ? Js[3 * j + c] : real(0);
        }
#pragma unroll
        for (int r = 0; r < RUN; ++r) {
          const int j = j0 + r;
          if (j >= L) continue;
          const real decay = pcoef_at(R, Ls, s, 0, f, j);
          const real cs = pcoef_at(R, Ls, s, 1, f, j);
          const real dre = pcoef_at(R, Ls, s, 4, f, j);
          real nj[3];
          if (R.magnetized) {
            const real sn = pcoef_at(R, Ls, s, 2, f, j);
            const real dpar = pcoef_at(R, Ls, s, 3, f, j);
            const real dim = pcoef_at(R, Ls, s, 5, f, j);
            real b[3];
            if (R.plasma_full) {
              const real* bp = R.bdir + 3 * ((size_t)f * L + j);
              b[0] = __ldg(bp);
              b[1] = __ldg(bp + 1);
              b[2] = __ldg(bp + 2);
            } else {
              b[0] = Ls.bd[3 * j];
              b[1] = Ls.bd[3 * j + 1];
              b[2] = Ls.bd[3 * j + 2];
            }
            const real eb = E[r][0] * b[0] + E[r][1] * b[1] + E[r][2] * b[2];
            real Ep[3], Eq[3], Ex[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              Ep[c] = eb * b[c];
              Eq[c] = E[r][c] - Ep[c];
            }
            Ex[0] = Eq[1] * b[2] - Eq[2] * b[1];
            Ex[1] = Eq[2] * b[0] - Eq[0] * b[2];
            Ex[2] = Eq[0] * b[1] - Eq[1] * b[0];
            const real jb = jv[r][0] * b[0] + jv[r][1] * b[1] + jv[r][2] * b[2];
            real Jp[3], Jq[3], Jx[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              Jp[c] = jb * b[c];
              Jq[c] = jv[r][c] - Jp[c];
            }
            Jx[0] = Jq[1] * b[2] - Jq[2] * b[1];
            Jx[1] = Jq[2] * b[0] - Jq[0] * b[2];
            Jx[2] = Jq[0] * b[1] - Jq[1] * b[0];
#pragma unroll
            for (int c = 0; c < 3; ++c)
              nj[c] = decay * Jp[c] + dpar * Ep[c] + decay * (cs * Jq[c] + sn * Jx[c]) + dre * Eq[c] + dim * Ex[c];
          } else {
#pragma unroll
            for (int c = 0; c < 3; ++c) nj[c] = decay * (cs * jv[r][c]) + dre * E[r][c];
          }
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            Js[3 * j + c] = nj[c];
            tot[r][c] += nj[c];
          }
        }
      }
      if (R.n_species > 1) {
        real* Jt = R.Jtot + ((size_t)f * L) * 3;
#pragma unroll
        for (int r = 0; r < RUN; ++r) {
          const int j = j0 + r;
          if (j < L) {
#pragma unroll
            for (int c = 0; c < 3; ++c) Jt[3 * j + c] = tot[r][c];
          }
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// E phase: Er (vertices x nodes) and Et (edges x midpoints).
// solver.py:923-989; plasma.py:503-527.
// ---------------------------------------------------------------------------
template <typename real, bool PLASMA, int RUN, int MAXDEG>
__global__ void __launch_bounds__(256) ke_kernel(const Rec<real>* __restrict__ recs, const int2* __restrict__ block_map,
                                                  int n_members, int istep) {
  extern __shared__ __align__(16) unsigned char dyn_smem[];
  __shared__ Rec<real> R;
  int member, patch;
  member_patch(block_map, n_members, member, patch);
  load_rec(R, recs + member);
  Layers<real> Ls;
  load_layers(R, reinterpret_cast<real*>(dyn_smem), Ls);
  const int L = R.L, Lp1 = L + 1;
  const int cn = (Lp1 + RUN - 1) / RUN, cm = (L + RUN - 1) / RUN;
  const uint32_t mag_cn = div_magic(cn), mag_cm = div_magic(cm);
  real* __restrict__ er = R.er;
  real* __restrict__ et = R.et;
  const real* __restrict__ ht = R.ht;
  const real* __restrict__ hr = R.hr;
  const real current = (R.n_src_er + R.n_src_et) > 0 ? (real)R.cur[istep] : real(0);
  const real* __restrict__ Jsum = PLASMA ? jsum(R) : nullptr;
  const bool full = R.full != 0;
  const bool coef_full = R.coef_full != 0;

  // ---- Er: dual-cell circulation of Ht, exponential loss, sources, Jr ----
  const int va = R.vptr[patch], vb = R.vptr[patch + 1];
  const int n_vert_items = (vb - va) * cn;
  for (int it = threadIdx.x; it < n_vert_items; it += blockDim.x) {
    const int vl = fast_div(it, mag_cn);
    const int k0 = (it - vl * cn) * RUN;
    const int slot = va + vl;
    const int v = __ldg(R.vlist + slot);
    real acc[RUN];
#pragma unroll
    for (int r = 0; r < RUN; ++r) acc[r] = real(0);
#pragma unroll
    for (int q = 0; q < MAXDEG; ++q) {
      const int e = __ldg(R.ps_edge + (size_t)slot * MAXDEG + q);
      const real c = __ldg(R.ps_coef + (size_t)slot * MAXDEG + q);
      const real* hrow = ht + (size_t)e * Lp1;
#pragma unroll
      for (int r = 0; r < RUN; ++r) {
        const int k = k0 + r;
        acc[r] += c * ((k < Lp1) ? hrow[k] : real(0));
      }
    }
    real* err = er + (size_t)v * Lp1;
    real ev[RUN];
#pragma unroll
    for (int r = 0; r < RUN; ++r) ev[r] = (k0 + r < Lp1) ? err[k0 + r] : real(0);
    real jr[RUN];
#pragma unroll
    for (int r = 0; r < RUN; ++r) jr[r] = real(0);
    if (PLASMA) {
      // radial plasma current at faces, area-averaged to the vertex, then to nodes
      real rav[RUN + 1];
#pragma unroll
      for (int r = 0; r <= RUN; ++r) rav[r] = real(0);
#pragma unroll 2
      for (int q = 0; q < MAXDEG; ++q) {
        const int f = __ldg(R.ps_face + (size_t)slot * MAXDEG + q);
        const real* wc = R.ps_wc + ((size_t)slot * MAXDEG + q) * 3;
        const real c0 = __ldg(wc), c1 = __ldg(wc + 1), c2 = __ldg(wc + 2);
        const real* jf = Jsum + (size_t)f * L * 3;
#pragma unroll
        for (int r = 0; r <= RUN; ++r) {
          int j = k0 - 1 + r;
          j = j < 0 ? 0 : (j >= L ? L - 1 : j);
          rav[r] += jf[3 * j] * c0 + jf[3 * j + 1] * c1 + jf[3 * j + 2] * c2;
        }
      }
#pragma unroll
      for (int r = 0; r < RUN; ++r) {
        const int k = k0 + r;
        jr[r] = (k == 0) ? rav[r + 1] : (k == L ? rav[r] : real(0.5) * (rav[r] + rav[r + 1]));
      }
    }
#pragma unroll
    for (int r = 0; r < RUN; ++r) {
      const int k = k0 + r;
      if (k >= Lp1) continue;
      const size_t o = (size_t)v * Lp1 + k;
      const real ca = coef_full ? __ldg(R.ca_er + o) : Ls.ca_er[k];
      const real cb = coef_full ? __ldg(R.cb_er + o) : Ls.cb_er[k];
      real x = ca * ev[r] + cb * (acc[r] * Ls.invr[k]);
      if (v >= R.src_er_vmin && v <= R.src_er_vmax) {
        for (int s = 0; s < R.n_src_er; ++s)
          if (__ldg(R.src_er_v + s) == v && __ldg(R.src_er_k + s) == k) x -= __ldg(R.src_er_c + s) * current;
      }
      if (PLASMA) x -= cb * jr[r];
      err[k] = x;
    }
  }

  // ---- Et: dual-edge difference of Hr minus (1/m) d(r Ht)/dr, loss, sources, Jt ----
  const int ea = R.eptr[patch], eb = R.eptr[patch + 1];
  const int n_edge_items = (eb - ea) * cm;
  for (int it = threadIdx.x; it < n_edge_items; it += blockDim.x) {
    const int el = fast_div(it, mag_cm);
    const int j0 = (it - el * cm) * RUN;
    const int e = ea + el;
    const int2 lr = __ldg(R.edge_lr + e);
    const real inv_p = __ldg(R.inv_phi + e);
    const real* hl = hr + (size_t)lr.x * L;
    const real* hq = hr + (size_t)lr.y * L;
    const real* htr = ht + (size_t)e * Lp1;
    real* etr = et + (size_t)e * L;
    real a[RUN], b[RUN], ev[RUN], hv[RUN + 1];
#pragma unroll
    for (int r = 0; r < RUN; ++r) {
      const int j = j0 + r;
      const bool ok = j < L;
      a[r] = ok ? hl[j] : real(0);
      b[r] = ok ? hq[j] : real(0);
      ev[r] = ok ? etr[j] : real(0);
    }
#pragma unroll
    for (int r = 0; r <= RUN; ++r) hv[r] = (j0 + r <= L) ? htr[j0 + r] : real(0);
    real jt[RUN];
#pragma unroll
    for (int r = 0; r < RUN; ++r) jt[r] = real(0);
    if (PLASMA) {
      const real* jl = Jsum + (size_t)lr.x * L * 3;
      const real* jq = Jsum + (size_t)lr.y * L * 3;
      const real* tl = R.tan_l + 3 * (size_t)e;
      const real* tq = R.tan_r + 3 * (size_t)e;
      const real l0 = __ldg(tl), l1 = __ldg(tl + 1), l2 = __ldg(tl + 2);
      const real q0 = __ldg(tq), q1 = __ldg(tq + 1), q2 = __ldg(tq + 2);
#pragma unroll
      for (int r = 0; r < RUN; ++r) {
        const int j = j0 + r < L ? j0 + r : L - 1;
        const real left = jl[3 * j] * l0 + jl[3 * j + 1] * l1 + jl[3 * j + 2] * l2;
        const real right = jq[3 * j] * q0 + jq[3 * j + 1] * q1 + jq[3 * j + 2] * q2;
        jt[r] = real(0.5) * (left + right);
      }
    }
#pragma unroll
    for (int r = 0; r < RUN; ++r) {
      const int j = j0 + r;
      if (j >= L) continue;
      real g = (a[r] - b[r]) * inv_p * Ls.invm[j];
      const real d = full ? (Ls.rr[j + 1] * hv[r + 1] - Ls.rr[j] * hv[r]) * Ls.invdr[j] * Ls.invm[j]
                          : (hv[r + 1] - hv[r]) * Ls.invdr[j];
      g -= d;
      const size_t o = (size_t)e * L + j;
      const real ca = coef_full ? __ldg(R.ca_et + o) : Ls.ca_et[j];
      const real cb = coef_full ? __ldg(R.cb_et + o) : Ls.cb_et[j];
      real x = ca * ev[r] + cb * g;
      if (e >= R.src_et_emin && e <= R.src_et_emax) {
        for (int s = 0; s < R.n_src_et; ++s)
          if (__ldg(R.src_et_e + s) == e && __ldg(R.src_et_j + s) == j) x -= __ldg(R.src_et_c + s) * current;
      }
      if (PLASMA) x -= cb * jt[r];
      etr[j] = x;
    }
  }
}

// ---------------------------------------------------------------------------
// Observation probe: one warp per row, lanes stride over the row's support
// points, float64 accumulation and a fixed-order shuffle reduction.
// ---------------------------------------------------------------------------
template <typename real>
__global__ void sample_kernel(const real* __restrict__ field, int pitch, int rows, int width,
                              const int* __restrict__ index, const int* __restrict__ layer,
                              const double* __restrict__ weight, double* __restrict__ out) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= rows) return;
  double acc = 0.0;
  for (int q = lane; q < width; q += 32) {
    const int o = warp * width + q;
    acc += weight[o] * (double)field[(size_t)index[o] * pitch + layer[o]];
  }
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) acc += __shfl_down_sync(0xFFFFFFFFu, acc, s);
  if (lane == 0) out[warp] = acc;
}

// Probe of the field named by ``kind`` in the launch record (0 er, 1 et, 2 hr,
// 3 ht): captured graphs read the current field pointer at run time.
template <typename real>
__global__ void sample_rec_kernel(const Rec<real>* __restrict__ rec, int kind, int rows, int width,
                                  const int* __restrict__ index, const int* __restrict__ layer,
                                  const double* __restrict__ weight, double* __restrict__ out) {
  const real* field = kind == 0 ? rec->er : kind == 1 ? rec->et : kind == 2 ? rec->hr : rec->ht;
  const int pitch = (kind == 0 || kind == 3) ? rec->L + 1 : rec->L;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= rows) return;
  double acc = 0.0;
  for (int q = lane; q < width; q += 32) {
    const int o = warp * width + q;
    acc += weight[o] * (double)field[(size_t)index[o] * pitch + layer[o]];
  }
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) acc += __shfl_down_sync(0xFFFFFFFFu, acc, s);
  if (lane == 0) out[warp] = acc;
}

// max |x| of up to four arrays; results combined with an order-independent
// atomic max on the bit pattern of non-negative doubles (NaN sorts above +Inf,
// so a non-finite field reports NaN or Inf).
template <typename real>
__global__ void max_abs_kernel(const real* __restrict__ a0, size_t n0, const real* __restrict__ a1, size_t n1,
                               const real* __restrict__ a2, size_t n2, const real* __restrict__ a3, size_t n3,
                               unsigned long long* __restrict__ out4) {
  const int which = blockIdx.y;
  const real* p = which == 0 ? a0 : which == 1 ? a1 : which == 2 ? a2 : a3;
  const size_t n = which == 0 ? n0 : which == 1 ? n1 : which == 2 ? n2 : n3;
  double m = 0.0;
  bool nan = false;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double v = fabs((double)p[i]);
    nan |= (v != v);
    m = fmax(m, v);
  }
  unsigned long long bits = nan ? 0x7FF8000000000000ull : (unsigned long long)__double_as_longlong(m);
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) {
    const unsigned long long o = __shfl_down_sync(0xFFFFFFFFu, bits, s);
    bits = o > bits ? o : bits;
  }
  if ((threadIdx.x & 31) == 0) atomicMax(out4 + which, bits);
}

// ---- ArrayBackend primitives on (N, cols) row-major arrays ----

// out[e] = x[pair.y] - x[pair.x] (head - tail), or x[pair.x] - x[pair.y] when
// first_minus_second (left face - right face).
template <typename real>
__global__ void pair_difference_kernel(const real* __restrict__ x, int cols, int nE, const int2* __restrict__ pair,
                                       bool first_minus_second, real* __restrict__ out) {
  const size_t n = (size_t)nE * cols;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int e = (int)(i / cols);
    const int c = (int)(i - (size_t)e * cols);
    const int2 t = pair[e];
    const int a = first_minus_second ? t.x : t.y;
    const int b = first_minus_second ? t.y : t.x;
    out[i] = x[(size_t)a * cols + c] - x[(size_t)b * cols + c];
  }
}

template <typename real>
__global__ void face_circulation_kernel(const real* __restrict__ x, int cols, int nF, const int4* __restrict__ fe,
                                        const int* __restrict__ fsign, real* __restrict__ out) {
  const size_t n = (size_t)nF * cols;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int f = (int)(i / cols);
    const int c = (int)(i - (size_t)f * cols);
    const int4 e = fe[f];
    const int* s = fsign + 3 * (size_t)f;
    real r = x[(size_t)e.x * cols + c] * (real)s[0];
    r += x[(size_t)e.y * cols + c] * (real)s[1];
    r += x[(size_t)e.z * cols + c] * (real)s[2];
    out[i] = r;
  }
}

template <typename real>
__global__ void dual_cell_circulation_kernel(const real* __restrict__ x, int cols, int nV, const int* __restrict__ off,
                                             const int* __restrict__ edge, const int* __restrict__ sign,
                                             real* __restrict__ out) {
  const size_t n = (size_t)nV * cols;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int v = (int)(i / cols);
    const int c = (int)(i - (size_t)v * cols);
    const int q0 = off[v], q1 = off[v + 1];
    real r = x[(size_t)edge[q0] * cols + c] * (real)sign[q0];
    for (int q = q0 + 1; q < q1; ++q) r += x[(size_t)edge[q] * cols + c] * (real)sign[q];
    out[i] = r;
  }
}

}  // namespace ifdtd
