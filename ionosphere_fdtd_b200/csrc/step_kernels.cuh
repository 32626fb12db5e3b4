// Device kernels of the geodesic FDTD time step (sm_100a).
//
// One launch record (Rec) describes one simulation: its device tables, its
// state pointers and the per-layer radial metric.  A CTA owns a "patch": a
// contiguous range of faces [f0, f0+fpp), the edges first met while scanning
// those faces (a contiguous edge range, because the reference numbers edges in
// face-scan order, mesh.py:674-708) and the vertices whose lowest-numbered
// incident face lies in the range (listed in vlist).  Inside a patch the work
// is flattened over (entity, radial layer) so a warp reads 32 consecutive
// radial samples of one column: every field access is a coalesced column
// segment.
//
// Two in-place launches form one leapfrog step, in the reference's order
// (solver.py:867-989):
//   kh_kernel: Ht (edges, nodes 0..L) with the lower surface-impedance ADE,
//              Hr (faces, midpoints) and the cold-plasma current ADE (faces).
//   ke_kernel: Er (vertices, nodes) and Et (edges, midpoints) with the
//              loss integrator, source injection and plasma current coupling.
// kh writes only H and plasma state and reads E; ke writes only E and reads H
// and the new plasma state, so both are race-free in place.  All sums run in a
// fixed order: results are bitwise repeatable.
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
  // vertex incidence (CSR, reference slot order)
  const int *v_off, *v_edge;
  const real* v_coef;    // sign * phi_e / A*_v
  // radial metric
  const real *invr, *rr, *mid, *invm, *invdr, *invcd;
  real dtmu;             // dt / mu0
  // loss coefficients
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
  const int *vf_off, *vf_face;
  const real* vf_wc;     // weight * face centre (3 per entry)
  const real *pcoef, *bdir;
};

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

// q = n / d for n < 2^24 and d <= 1024 with m = ceil(2^32 / d).
__device__ __forceinline__ int fast_div(int n, uint32_t m) {
  return (int)__umulhi((uint32_t)n, m);
}

template <typename real>
__device__ __forceinline__ real plasma_coef(const Rec<real>& R, int s, int c, int f, int j) {
  const size_t rows = R.plasma_full ? (size_t)R.nF : 1;
  const size_t row = R.plasma_full ? (size_t)f : 0;
  return __ldg(R.pcoef + (((size_t)(s * 6 + c) * rows + row) * R.L + j));
}

// ---------------------------------------------------------------------------
// H phase: Ht (edges x nodes), surface-impedance ADE, Hr (faces x midpoints),
// cold-plasma current ADE (faces x midpoints).
// solver.py:877-921; surface_impedance.py:225-270; plasma.py:413-442, 489-501.
// ---------------------------------------------------------------------------
template <typename real, bool PLASMA>
__global__ void __launch_bounds__(256) kh_kernel(const Rec<real>* __restrict__ recs,
                                                  const int2* __restrict__ block_map,
                                                  int n_members) {
  __shared__ Rec<real> R;
  int member = 0, patch = blockIdx.x;
  if (n_members > 1) {
    const int2 bm = block_map[blockIdx.x];
    member = bm.x;
    patch = bm.y;
  }
  load_rec(R, recs + member);
  const int L = R.L, Lp1 = L + 1;
  const uint32_t mag_n = 0xFFFFFFFFu / (uint32_t)Lp1 + 1u;
  const uint32_t mag_m = 0xFFFFFFFFu / (uint32_t)L + 1u;
  const real* __restrict__ er = R.er;
  const real* __restrict__ et = R.et;
  real* __restrict__ ht = R.ht;
  real* __restrict__ hr = R.hr;
  const real dtmu = R.dtmu;

  // ---- Ht: d/dt Ht = (grad_s Er - (1/r) d(m Et)/dr) / mu0 with PEC ghosts ----
  const int ea = R.eptr[patch], eb = R.eptr[patch + 1];
  const int n_edge_el = (eb - ea) * Lp1;
  const bool si = R.si_terms > 0;
  for (int i = threadIdx.x; i < n_edge_el; i += blockDim.x) {
    const int el = fast_div(i, mag_n);
    const int k = i - el * Lp1;
    if (si && k == 0) continue;  // the surface ADE owns the lowest plane
    const int e = ea + el;
    const int2 th = __ldg(R.edge_th + e);
    real g = (er[(size_t)th.y * Lp1 + k] - er[(size_t)th.x * Lp1 + k]) * __ldg(R.inv_theta + e);
    g *= __ldg(R.invr + k);
    const real* etr = et + (size_t)e * L;
    real up = (k < L) ? etr[k] : real(0);
    real dn = (k > 0) ? etr[k - 1] : real(0);
    real d;
    if (R.full) {
      if (k < L) up *= __ldg(R.mid + k);
      if (k > 0) dn *= __ldg(R.mid + k - 1);
      d = (up - dn) * __ldg(R.invcd + k) * __ldg(R.invr + k);
    } else {
      d = (up - dn) * __ldg(R.invcd + k);
    }
    ht[(size_t)e * Lp1 + k] += (g - d) * dtmu;
  }

  // ---- lower surface-impedance boundary (implicit, trapezoidal ADE) ----
  if (si) {
    const int T = R.si_terms;
    for (int el = threadIdx.x; el < eb - ea; el += blockDim.x) {
      const int e = ea + el;
      const int2 th = __ldg(R.edge_th + e);
      const real h_old = ht[(size_t)e * Lp1];
      real g0 = (er[(size_t)th.y * Lp1] - er[(size_t)th.x * Lp1]) * __ldg(R.inv_theta + e);
      g0 *= __ldg(R.invr);
      const real e1 = R.si_metric * et[(size_t)e * L];
      const real s = __ldg(R.si_scale + e);
      real* mem = R.si_mem + (size_t)e * T;
      real hist = real(0);
      for (int p = 0; p < T; ++p) hist += mem[p] * __ldg(R.si_hist + p);
      hist *= s;
      const real kap = R.si_kappa;
      const real c = kap * (s * R.si_hist_sum);
      const real h_new =
          ((real(1) - real(0.5) * c) * h_old + dtmu * g0 - kap * e1 + kap * hist) /
          (real(1) + real(0.5) * c);
      ht[(size_t)e * Lp1] = h_new;
      const real hs = h_new + h_old;
      for (int p = 0; p < T; ++p) mem[p] = mem[p] * __ldg(R.si_decay + p) + hs * __ldg(R.si_drive + p);
    }
  }

  // ---- Hr and the plasma current on owned faces ----
  const int fa = patch * R.fpp;
  const int fb = min(fa + R.fpp, R.nF);
  const int n_face_el = (fb - fa) * L;
  for (int i = threadIdx.x; i < n_face_el; i += blockDim.x) {
    const int fl = fast_div(i, mag_m);
    const int j = i - fl * L;
    const int f = fa + fl;
    const int4 fe = __ldg(R.face_e + f);
    const real e0 = et[(size_t)fe.x * L + j];
    const real e1 = et[(size_t)fe.y * L + j];
    const real e2 = et[(size_t)fe.z * L + j];
    const real* w = R.face_w + 3 * (size_t)f;
    const real circ = __ldg(w) * e0 + __ldg(w + 1) * e1 + __ldg(w + 2) * e2;
    hr[(size_t)f * L + j] -= circ * __ldg(R.invm + j) * dtmu;
    if (PLASMA) {
      const int4 fv = __ldg(R.face_v + f);
      const real third = real(1) / real(3);
      const real n0 = (er[(size_t)fv.x * Lp1 + j] + er[(size_t)fv.y * Lp1 + j] + er[(size_t)fv.z * Lp1 + j]) * third;
      const real n1 = (er[(size_t)fv.x * Lp1 + j + 1] + er[(size_t)fv.y * Lp1 + j + 1] + er[(size_t)fv.z * Lp1 + j + 1]) * third;
      const real rad = real(0.5) * (n0 + n1);
      const real* rc = R.recon + 9 * (size_t)f;
      const real* cf = R.centre + 3 * (size_t)f;
      real E[3];
#pragma unroll
      for (int c = 0; c < 3; ++c)
        E[c] = e0 * __ldg(rc + c) + e1 * __ldg(rc + 3 + c) + e2 * __ldg(rc + 6 + c) + rad * __ldg(cf + c);
      real b[3] = {real(0), real(0), real(0)};
      real Ep[3], Eq[3], Ex[3];  // parallel, perpendicular, perpendicular x b
      if (R.magnetized) {
        const real* bp = R.bdir + 3 * (R.plasma_full ? ((size_t)f * L + j) : (size_t)j);
        b[0] = __ldg(bp);
        b[1] = __ldg(bp + 1);
        b[2] = __ldg(bp + 2);
        const real eb = E[0] * b[0] + E[1] * b[1] + E[2] * b[2];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          Ep[c] = eb * b[c];
          Eq[c] = E[c] - Ep[c];
        }
        Ex[0] = Eq[1] * b[2] - Eq[2] * b[1];
        Ex[1] = Eq[2] * b[0] - Eq[0] * b[2];
        Ex[2] = Eq[0] * b[1] - Eq[1] * b[0];
      }
      real tot[3] = {real(0), real(0), real(0)};
      const size_t jo = ((size_t)f * L + j) * 3;
      for (int s = 0; s < R.n_species; ++s) {
        real* Js = R.J[s] + jo;
        const real decay = plasma_coef(R, s, 0, f, j);
        const real cs = plasma_coef(R, s, 1, f, j);
        const real dre = plasma_coef(R, s, 4, f, j);
        real nj[3];
        if (R.magnetized) {
          const real sn = plasma_coef(R, s, 2, f, j);
          const real dpar = plasma_coef(R, s, 3, f, j);
          const real dim = plasma_coef(R, s, 5, f, j);
          const real J0 = Js[0], J1 = Js[1], J2 = Js[2];
          const real jb = J0 * b[0] + J1 * b[1] + J2 * b[2];
          real Jp[3], Jq[3], Jx[3];
          Jp[0] = jb * b[0]; Jp[1] = jb * b[1]; Jp[2] = jb * b[2];
          Jq[0] = J0 - Jp[0]; Jq[1] = J1 - Jp[1]; Jq[2] = J2 - Jp[2];
          Jx[0] = Jq[1] * b[2] - Jq[2] * b[1];
          Jx[1] = Jq[2] * b[0] - Jq[0] * b[2];
          Jx[2] = Jq[0] * b[1] - Jq[1] * b[0];
#pragma unroll
          for (int c = 0; c < 3; ++c)
            nj[c] = decay * Jp[c] + dpar * Ep[c] + decay * (cs * Jq[c] + sn * Jx[c]) + dre * Eq[c] + dim * Ex[c];
        } else {
#pragma unroll
          for (int c = 0; c < 3; ++c) nj[c] = decay * (cs * Js[c]) + dre * E[c];
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          Js[c] = nj[c];
          tot[c] += nj[c];
        }
      }
      if (R.n_species > 1) {
#pragma unroll
        for (int c = 0; c < 3; ++c) R.Jtot[jo + c] = tot[c];
      }
    }
  }
}

// Summed plasma current at (face, midpoint): species 0 directly, else Jtot.
template <typename real>
__device__ __forceinline__ const real* jsum(const Rec<real>& R) {
  return R.n_species > 1 ? R.Jtot : R.J[0];
}

// ---------------------------------------------------------------------------
// E phase: Er (vertices x nodes) and Et (edges x midpoints).
// solver.py:923-989; plasma.py:503-527.
// ---------------------------------------------------------------------------
template <typename real, bool PLASMA>
__global__ void __launch_bounds__(256) ke_kernel(const Rec<real>* __restrict__ recs,
                                                  const int2* __restrict__ block_map,
                                                  int n_members, int istep) {
  __shared__ Rec<real> R;
  int member = 0, patch = blockIdx.x;
  if (n_members > 1) {
    const int2 bm = block_map[blockIdx.x];
    member = bm.x;
    patch = bm.y;
  }
  load_rec(R, recs + member);
  const int L = R.L, Lp1 = L + 1;
  const uint32_t mag_n = 0xFFFFFFFFu / (uint32_t)Lp1 + 1u;
  const uint32_t mag_m = 0xFFFFFFFFu / (uint32_t)L + 1u;
  real* __restrict__ er = R.er;
  real* __restrict__ et = R.et;
  const real* __restrict__ ht = R.ht;
  const real* __restrict__ hr = R.hr;
  const real current = (R.n_src_er + R.n_src_et) > 0 ? (real)R.cur[istep] : real(0);
  const real* Jt = PLASMA ? jsum(R) : nullptr;

  // ---- Er: dual-cell circulation of Ht, exponential loss, sources, Jr ----
  const int va = R.vptr[patch], vb = R.vptr[patch + 1];
  const int n_vert_el = (vb - va) * Lp1;
  for (int i = threadIdx.x; i < n_vert_el; i += blockDim.x) {
    const int vl = fast_div(i, mag_n);
    const int k = i - vl * Lp1;
    const int v = __ldg(R.vlist + va + vl);
    const int q0 = __ldg(R.v_off + v), q1 = __ldg(R.v_off + v + 1);
    real acc = real(0);
    for (int q = q0; q < q1; ++q) acc += __ldg(R.v_coef + q) * ht[(size_t)__ldg(R.v_edge + q) * Lp1 + k];
    acc *= __ldg(R.invr + k);
    const size_t o = (size_t)v * Lp1 + k;
    const real ca = R.coef_full ? __ldg(R.ca_er + o) : __ldg(R.ca_er + k);
    const real cb = R.coef_full ? __ldg(R.cb_er + o) : __ldg(R.cb_er + k);
    real x = ca * er[o] + cb * acc;
    if (v >= R.src_er_vmin && v <= R.src_er_vmax) {
      for (int s = 0; s < R.n_src_er; ++s)
        if (__ldg(R.src_er_v + s) == v && __ldg(R.src_er_k + s) == k) x -= __ldg(R.src_er_c + s) * current;
    }
    if (PLASMA) {
      const int p0 = __ldg(R.vf_off + v), p1 = __ldg(R.vf_off + v + 1);
      const int jlo = (k == 0) ? 0 : k - 1;
      const int jhi = (k == L) ? L - 1 : k;
      real lo = real(0), hi = real(0);
      for (int p = p0; p < p1; ++p) {
        const size_t fo = (size_t)__ldg(R.vf_face + p) * L;
        const real* wc = R.vf_wc + 3 * (size_t)p;
        const real* a = Jt + (fo + jlo) * 3;
        lo += a[0] * __ldg(wc) + a[1] * __ldg(wc + 1) + a[2] * __ldg(wc + 2);
        if (jhi != jlo) {
          const real* c = Jt + (fo + jhi) * 3;
          hi += c[0] * __ldg(wc) + c[1] * __ldg(wc + 1) + c[2] * __ldg(wc + 2);
        }
      }
      const real jr = (jhi != jlo) ? real(0.5) * (lo + hi) : lo;
      x -= cb * jr;
    }
    er[o] = x;
  }

  // ---- Et: dual-edge difference of Hr minus (1/m) d(r Ht)/dr, loss, sources, Jt ----
  const int ea = R.eptr[patch], eb = R.eptr[patch + 1];
  const int n_edge_el = (eb - ea) * L;
  for (int i = threadIdx.x; i < n_edge_el; i += blockDim.x) {
    const int el = fast_div(i, mag_m);
    const int j = i - el * L;
    const int e = ea + el;
    const int2 lr = __ldg(R.edge_lr + e);
    real g = (hr[(size_t)lr.x * L + j] - hr[(size_t)lr.y * L + j]) * __ldg(R.inv_phi + e);
    g *= __ldg(R.invm + j);
    const real* htr = ht + (size_t)e * Lp1;
    real d;
    if (R.full)
      d = (__ldg(R.rr + j + 1) * htr[j + 1] - __ldg(R.rr + j) * htr[j]) * __ldg(R.invdr + j) * __ldg(R.invm + j);
    else
      d = (htr[j + 1] - htr[j]) * __ldg(R.invdr + j);
    g -= d;
    const size_t o = (size_t)e * L + j;
    const real ca = R.coef_full ? __ldg(R.ca_et + o) : __ldg(R.ca_et + j);
    const real cb = R.coef_full ? __ldg(R.cb_et + o) : __ldg(R.cb_et + j);
    real x = ca * et[o] + cb * g;
    if (e >= R.src_et_emin && e <= R.src_et_emax) {
      for (int s = 0; s < R.n_src_et; ++s)
        if (__ldg(R.src_et_e + s) == e && __ldg(R.src_et_j + s) == j) x -= __ldg(R.src_et_c + s) * current;
    }
    if (PLASMA) {
      const real* a = Jt + ((size_t)lr.x * L + j) * 3;
      const real* c = Jt + ((size_t)lr.y * L + j) * 3;
      const real* tl = R.tan_l + 3 * (size_t)e;
      const real* tr = R.tan_r + 3 * (size_t)e;
      const real left = a[0] * __ldg(tl) + a[1] * __ldg(tl + 1) + a[2] * __ldg(tl + 2);
      const real right = c[0] * __ldg(tr) + c[1] * __ldg(tr + 1) + c[2] * __ldg(tr + 2);
      x -= cb * (real(0.5) * (left + right));
    }
    et[o] = x;
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
  const real* src[4] = {a0, a1, a2, a3};
  const size_t len[4] = {n0, n1, n2, n3};
  const int which = blockIdx.y;
  const real* p = src[which];
  const size_t n = len[which];
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
