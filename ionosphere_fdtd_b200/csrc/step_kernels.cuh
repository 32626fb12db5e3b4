// Device kernels of the geodesic FDTD time step (sm_100a).
//
// One launch record (Rec) describes one simulation: its device tables, its
// state pointers and the per-layer radial metric.  A CTA owns a "patch": a
// contiguous range of faces [f0, f0+fpp), the edges first met while scanning
// those faces (a contiguous edge range, because the reference numbers edges in
// face-scan order, mesh.py:674-708) and the vertices whose lowest-numbered
// incident face lies in the range (listed in vlist).
//
// Layout: rows of node arrays (er, ht) have pitch Pn >= L+1 and rows of
// midpoint arrays (et, hr, plasma current components) pitch Pm >= L, both
// multiples of 16 bytes, with zero padding that every kernel keeps zero.  A
// thread owns one 16-byte run (4 floats or 2 doubles) of one column, so each
// access to a gathered neighbour column is one aligned vector load and a warp
// reads 512 contiguous bytes per column segment.  Per-entity tables are packed
// for vector loads; vertex gathers use fixed-width slot tables (MAXDEG slots,
// padded with coefficient 0 as the reference pads its incidence table,
// torch_backend.py:66-89) stored in patch order, so index chains are two loads
// deep and all gathers unroll.  Per-layer metric factors and altitude-only
// coefficient rows are staged in shared memory.
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
constexpr int kMaxSources = 16;

template <typename real>
struct Rec {
  // sizes and switches
  int nV, nE, nF, L, Pn, Pm;
  int n_patches_h, fpp_h, n_patches_e, fpp_e;
  int full, si_terms, n_species, plasma_full, magnetized, coef_full;
  // 1: the plasma current is held in face frames while the kernels run
  // (component 0 along the face centre, 1 and 2 in the face's tangent plane);
  // the reconstruction rows, vertex weights and edge tangents are then in the
  // same frames and packed as the local runs read them
  int plasma_local;
  int n_src_er, n_src_et;
  int maxdeg, slot_width, layer_reals;
  // state
  real *er, *et, *hr, *ht, *si_mem;
  real* J[kMaxSpecies];  // (F, 3, Pm) per species
  real* Jtot;            // summed species current when n_species > 1
  const double* cur;     // per-step source current (staging row)
  int* status;           // device status word (bit 0: a staging wait timed out)
  // ownership: H phase patches own faces [p*fpp_h, ...) and eptr_h edges;
  // E phase patches own vertices vlist[vptr[p]..] and eptr_e edges
  const int *eptr_h, *eptr_e, *vptr, *vlist;
  // edges
  const int2 *edge_th, *edge_lr;
  const real *inv_theta, *inv_phi;
  const real* tan;       // (E, 8): left tangent, 0, right tangent, 0
  // faces
  const int4 *face_e, *face_v;
  const real* face_w;    // (F, 4): sign_i * theta_i / A_f, 0
  const real* face_pl;   // (F, 12): reconstruction row i then centre component i
  const real* frame;     // (F, 12): face-frame rows e0, 0, e1, 0, e2, 0 (plasma_local only)
  // vertex slots in vlist order, slot_width entries per vertex
  const int* ps_edge;
  const real* ps_coef;   // sign * phi_e / A*_v, 0 in padding slots
  const int* ps_face;
  const real* ps_wc;     // (V, slot_width, 4): area weight * face centre, 0 in padding slots
  // pipelined kernels: per patch copy descriptors (dptr: CSR offsets into desc)
  // and the per-patch table blobs they copy (16-byte units)
  const int *dptr_h, *dptr_e;
  const int4 *desc_h, *desc_e;
  const unsigned char *tab_h, *tab_e;
  // radial metric rows (padded; staged in shared memory by the kernels)
  const real *invr, *rr, *mid, *invm, *invdr, *invcd;
  // fused per-layer rows: H-edge (hA, hU, hD), H-face (hC), E-vertex current
  // weights (vwl, vwu), E-edge radial curl (eU, eD); zero beyond the grid
  const real *hA, *hU, *hD, *hC, *vwl, *vwu, *eU, *eD;
  real dtmu;             // dt / mu0
  // loss coefficients: (rows, Pn) / (rows, Pm), rows = 1 or V / E
  const real *ca_er, *cb_er, *ca_et, *cb_et;
  // sources (supports listed inline: the record lives in shared memory)
  int src_er_v[kMaxSources], src_er_k[kMaxSources], src_et_e[kMaxSources], src_et_j[kMaxSources];
  real src_er_c[kMaxSources], src_et_c[kMaxSources];
  // surface impedance
  real si_metric, si_kappa, si_hist_sum;
  const real *si_scale, *si_decay, *si_drive, *si_hist;
  // plasma: coefficients (S, 6, rows, Pm), unit B (rows, 3, Pm)
  const real *pcoef, *bdir;
};

template <typename real>
struct Lanes;
template <>
struct Lanes<float> {
  static constexpr int N = 4;
};
template <>
struct Lanes<double> {
  static constexpr int N = 2;
};

// One 16-byte radial run.
template <typename real>
struct Run {
  real x[Lanes<real>::N];
};

template <typename real>
__device__ __forceinline__ Run<real> ld16(const real* p) {
  Run<real> r;
  if constexpr (sizeof(real) == 4) {
    const float4 t = *reinterpret_cast<const float4*>(p);
    r.x[0] = t.x; r.x[1] = t.y; r.x[2] = t.z; r.x[3] = t.w;
  } else {
    const double2 t = *reinterpret_cast<const double2*>(p);
    r.x[0] = t.x; r.x[1] = t.y;
  }
  return r;
}

// Read-only (non-coherent) variant for arrays the kernel does not write.
template <typename real>
__device__ __forceinline__ Run<real> ldg16(const real* p) {
  Run<real> r;
  if constexpr (sizeof(real) == 4) {
    const float4 t = __ldg(reinterpret_cast<const float4*>(p));
    r.x[0] = t.x; r.x[1] = t.y; r.x[2] = t.z; r.x[3] = t.w;
  } else {
    const double2 t = __ldg(reinterpret_cast<const double2*>(p));
    r.x[0] = t.x; r.x[1] = t.y;
  }
  return r;
}

// Four consecutive reals from a 16-byte aligned address (one or two vector loads).
template <typename real>
__device__ __forceinline__ void ld4(const real* p, real (&v)[4]) {
  if constexpr (sizeof(real) == 4) {
    const float4 t = *reinterpret_cast<const float4*>(p);
    v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
  } else {
    const double2 a = *reinterpret_cast<const double2*>(p), b = *reinterpret_cast<const double2*>(p + 2);
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
  }
}

// Four consecutive reals to a 16-byte aligned global address.
template <typename real>
__device__ __forceinline__ void st4(real* p, const real (&v)[4]) {
  if constexpr (sizeof(real) == 4) {
    __stcg(reinterpret_cast<float4*>(p), make_float4(v[0], v[1], v[2], v[3]));
  } else {
    __stcg(reinterpret_cast<double2*>(p), make_double2(v[0], v[1]));
    __stcg(reinterpret_cast<double2*>(p + 2), make_double2(v[2], v[3]));
  }
}

template <typename real>
__device__ __forceinline__ Run<real> zero_run() {
  Run<real> r;
#pragma unroll
  for (int i = 0; i < Lanes<real>::N; ++i) r.x[i] = real(0);
  return r;
}

// 16-byte store to global memory (outputs are always global; the explicit
// global store also tells the compiler it cannot alias shared memory).
template <typename real>
__device__ __forceinline__ void st16(real* p, const Run<real>& r) {
  if constexpr (sizeof(real) == 4) {
    __stcg(reinterpret_cast<float4*>(p), make_float4(r.x[0], r.x[1], r.x[2], r.x[3]));
  } else {
    __stcg(reinterpret_cast<double2*>(p), make_double2(r.x[0], r.x[1]));
  }
}

// Shared-memory view of the per-layer rows of one record.
template <typename real>
struct Layers {
  real *invr, *rr, *invcd, *mid, *invm, *invdr;
  real *hA, *hU, *hD, *vwl, *vwu, *hC, *eU, *eD;
  real *ca_er, *cb_er, *ca_et, *cb_et;  // compressed coefficient rows (else null)
  real *pc, *bd;                        // compressed plasma rows (else null)
  real *si_decay, *si_drive, *si_hist;  // surface-impedance pole rows (else null)
};

// Number of reals of per-layer data staged in shared memory (host and device).
__host__ __device__ inline int layer_reals(int Pn, int Pm, int coef_full, int species, int plasma_full, int magnetized,
                                           int si_terms) {
  int n = 8 * Pn + 6 * Pm;
  if (!coef_full) n += 2 * Pn + 2 * Pm;
  if (species > 0 && !plasma_full) n += 6 * species * Pm + (magnetized ? 3 * Pm : 0);
  n += 3 * si_terms;
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
  const int Pn = R.Pn, Pm = R.Pm;
  real* p = smem;
  Ls.invr = p; p += Pn;
  Ls.rr = p; p += Pn;
  Ls.invcd = p; p += Pn;
  Ls.mid = p; p += Pm;
  Ls.invm = p; p += Pm;
  Ls.invdr = p; p += Pm;
  copy_row(Ls.invr, R.invr, Pn);
  copy_row(Ls.rr, R.rr, Pn);
  copy_row(Ls.invcd, R.invcd, Pn);
  copy_row(Ls.mid, R.mid, Pm);
  copy_row(Ls.invm, R.invm, Pm);
  copy_row(Ls.invdr, R.invdr, Pm);
  Ls.hA = p; p += Pn;
  Ls.hU = p; p += Pn;
  Ls.hD = p; p += Pn;
  Ls.vwl = p; p += Pn;
  Ls.vwu = p; p += Pn;
  Ls.hC = p; p += Pm;
  Ls.eU = p; p += Pm;
  Ls.eD = p; p += Pm;
  copy_row(Ls.hA, R.hA, Pn);
  copy_row(Ls.hU, R.hU, Pn);
  copy_row(Ls.hD, R.hD, Pn);
  copy_row(Ls.vwl, R.vwl, Pn);
  copy_row(Ls.vwu, R.vwu, Pn);
  copy_row(Ls.hC, R.hC, Pm);
  copy_row(Ls.eU, R.eU, Pm);
  copy_row(Ls.eD, R.eD, Pm);
  Ls.ca_er = Ls.cb_er = Ls.ca_et = Ls.cb_et = nullptr;
  if (!R.coef_full) {
    Ls.ca_er = p; p += Pn;
    Ls.cb_er = p; p += Pn;
    Ls.ca_et = p; p += Pm;
    Ls.cb_et = p; p += Pm;
    copy_row(Ls.ca_er, R.ca_er, Pn);
    copy_row(Ls.cb_er, R.cb_er, Pn);
    copy_row(Ls.ca_et, R.ca_et, Pm);
    copy_row(Ls.cb_et, R.cb_et, Pm);
  }
  Ls.pc = Ls.bd = nullptr;
  if (R.n_species > 0 && !R.plasma_full) {
    Ls.pc = p; p += 6 * R.n_species * Pm;
    copy_row(Ls.pc, R.pcoef, 6 * R.n_species * Pm);
    if (R.magnetized) {
      Ls.bd = p; p += 3 * Pm;
      copy_row(Ls.bd, R.bdir, 3 * Pm);
    }
  }
  Ls.si_decay = Ls.si_drive = Ls.si_hist = nullptr;
  if (R.si_terms > 0) {
    Ls.si_decay = p; p += R.si_terms;
    Ls.si_drive = p; p += R.si_terms;
    Ls.si_hist = p; p += R.si_terms;
    copy_row(Ls.si_decay, R.si_decay, R.si_terms);
    copy_row(Ls.si_drive, R.si_drive, R.si_terms);
    copy_row(Ls.si_hist, R.si_hist, R.si_terms);
  }
  __syncthreads();
}

// q = n / d for n < 2^24 and 1 <= d <= 1024 with m = ceil(2^32 / d); d = 1
// (m = 2^32 does not fit) is encoded as m = 0 and divides as the identity.
__device__ __forceinline__ int fast_div(int n, uint32_t m) { return m ? (int)__umulhi((uint32_t)n, m) : n; }
__device__ __forceinline__ uint32_t div_magic(int d) { return d == 1 ? 0u : 0xFFFFFFFFu / (uint32_t)d + 1u; }

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
// Per-run arithmetic shared by the direct and the pipelined kernels.  Input
// row pointers and per-entity table pointers may address shared or global
// memory; outputs are global.  Radial factors come from fused per-layer rows
// (host-computed in float64, zero beyond the last node or midpoint) loaded as
// 16-byte vectors, so padding lanes come out zero without per-element tests.
// ---------------------------------------------------------------------------

// acc + (x*c0 + y*c1 + z*c2) with explicit roundings, so every kernel that
// accumulates a vertex's radial current gets the same bits.
__device__ __forceinline__ float rav_term(float acc, float x, float y, float z, float c0, float c1, float c2) {
  float t = __fmul_rn(x, c0);
  t = __fmaf_rn(y, c1, t);
  t = __fmaf_rn(z, c2, t);
  return __fadd_rn(acc, t);
}
__device__ __forceinline__ double rav_term(double acc, double x, double y, double z, double c0, double c1, double c2) {
  double t = __dmul_rn(x, c0);
  t = __fma_rn(y, c1, t);
  t = __fma_rn(z, c2, t);
  return __dadd_rn(acc, t);
}

// Radial current of one vertex at midpoints j0..j0+N-1: sum over its face
// slots of (area weight * face centre) . J (plasma.py:511-526).
template <typename real, int MAXDEG>
__device__ __forceinline__ Run<real> vertex_radial_current(const real* const* jrows, const real* wcs, int j0, int Pm) {
  constexpr int N = Lanes<real>::N;
  Run<real> acc = zero_run<real>();
#pragma unroll
  for (int q = 0; q < MAXDEG; ++q) {
    real wc[4];
    ld4(wcs + 4 * q, wc);
    const real* jf = jrows[q];
    const Run<real> jx = ld16(jf + j0), jy = ld16(jf + Pm + j0), jz = ld16(jf + 2 * Pm + j0);
#pragma unroll
    for (int r = 0; r < N; ++r) acc.x[r] = rav_term(acc.x[r], jx.x[r], jy.x[r], jz.x[r], wc[0], wc[1], wc[2]);
  }
  return acc;
}

// Radial current of one vertex at the single midpoint j (the same rav_term
// sequence over the slots as vertex_radial_current, so the same bits).
template <typename real, int MAXDEG>
__device__ __forceinline__ real vertex_radial_current_at(const real* const* jrows, const real* wcs, int j, int Pm) {
  real acc = real(0);
#pragma unroll
  for (int q = 0; q < MAXDEG; ++q) {
    real wc[4];
    ld4(wcs + 4 * q, wc);
    const real* jf = jrows[q];
    acc = rav_term(acc, jf[j], jf[Pm + j], jf[2 * Pm + j], wc[0], wc[1], wc[2]);
  }
  return acc;
}

// Face-frame radial current of one vertex at midpoints j0..j0+N-1: sum over
// its face slots of weight_q * J_r (component 0 of the face's current, the
// component along the face centre), wq[q] = area weight * |face centre| of slot
// q (zero in padding slots).  The terms the face frame makes zero (the
// tangential components against a zero weight) are not formed.
__device__ __forceinline__ float rav_local(float acc, float x, float w) { return __fadd_rn(acc, __fmul_rn(x, w)); }
__device__ __forceinline__ double rav_local(double acc, double x, double w) { return __dadd_rn(acc, __dmul_rn(x, w)); }

template <typename real, int MAXDEG>
__device__ __forceinline__ void slot_weights(const real* wq, real (&w)[(MAXDEG + 3) / 4 * 4]) {
#pragma unroll
  for (int q = 0; q < MAXDEG; q += 4) {
    real c4[4];
    ld4(wq + q, c4);
#pragma unroll
    for (int i = 0; i < 4; ++i) w[q + i] = c4[i];
  }
}

template <typename real, int MAXDEG>
__device__ __forceinline__ Run<real> vertex_radial_current_local(const real* const* jrows, const real* wq, int j0) {
  constexpr int N = Lanes<real>::N;
  real w[(MAXDEG + 3) / 4 * 4];
  slot_weights<real, MAXDEG>(wq, w);
  Run<real> acc = zero_run<real>();
#pragma unroll
  for (int q = 0; q < MAXDEG; ++q) {
    const Run<real> jr = ld16(jrows[q] + j0);
#pragma unroll
    for (int r = 0; r < N; ++r) acc.x[r] = rav_local(acc.x[r], jr.x[r], w[q]);
  }
  return acc;
}

// The same sum at the single midpoint j (same sequence, same bits).
template <typename real, int MAXDEG>
__device__ __forceinline__ real vertex_radial_current_local_at(const real* const* jrows, const real* wq, int j) {
  real w[(MAXDEG + 3) / 4 * 4];
  slot_weights<real, MAXDEG>(wq, w);
  real acc = real(0);
#pragma unroll
  for (int q = 0; q < MAXDEG; ++q) acc = rav_local(acc, jrows[q][j], w[q]);
  return acc;
}

// Source supports matching entity `id` exist (one pass over the record's list).
__device__ __forceinline__ bool source_hit(const int* ids, int n, int id) {
  bool hit = false;
  for (int s = 0; s < n; ++s) hit |= ids[s] == id;
  return hit;
}

// ---- surface-impedance ADE pieces (surface_impedance.py:225-270) ----
// History sum of four poles: explicit fused multiply-adds in pole order.
__device__ __forceinline__ float si_quad(const float* m, const float* w) {
  float m4[4], w4[4];
  ld4(m, m4);
  ld4(w, w4);
  float a = __fmul_rn(m4[0], w4[0]);
  a = __fmaf_rn(m4[1], w4[1], a);
  a = __fmaf_rn(m4[2], w4[2], a);
  return __fmaf_rn(m4[3], w4[3], a);
}
__device__ __forceinline__ double si_quad(const double* m, const double* w) {
  double m4[4], w4[4];
  ld4(m, m4);
  ld4(w, w4);
  double a = __dmul_rn(m4[0], w4[0]);
  a = __fma_rn(m4[1], w4[1], a);
  a = __fma_rn(m4[2], w4[2], a);
  return __fma_rn(m4[3], w4[3], a);
}
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }

// Pole history sum: quads of four poles, added in pole order (the order the
// four-lane pass reproduces); poles one by one when T is not a multiple of 4.
template <typename real>
__device__ __forceinline__ real si_history(const real* mem, const real* w, int T) {
  if ((T & 3) == 0) {
    real h = si_quad(mem, w);
    for (int p = 4; p < T; p += 4) h = add_rn(h, si_quad(mem + p, w + p));
    return h;
  }
  real h = real(0);
  for (int p = 0; p < T; ++p) h += mem[p] * w[p];
  return h;
}

// New node-0 Ht from the old value, the surface gradient term g0, the Et term
// e1, the edge's scale s and the pole history sum.
template <typename real>
__device__ __forceinline__ real si_boundary(const Rec<real>& R, real h_old, real g0, real e1, real s, real hist) {
  hist *= s;
  const real kap = R.si_kappa;
  const real c = kap * (s * R.si_hist_sum);
  return ((real(1) - real(0.5) * c) * h_old + R.dtmu * g0 - kap * e1 + kap * hist) / (real(1) + real(0.5) * c);
}

// Poles p..p+3 of the memory: mem = mem * decay + (h_new + h_old) * drive.
template <typename real>
__device__ __forceinline__ void si_update_quad(const real* in, real* out, const Layers<real>& Ls, int p, real hs) {
  real m4[4], d4[4], r4[4];
  ld4(in, m4);
  ld4(Ls.si_decay + p, d4);
  ld4(Ls.si_drive + p, r4);
#pragma unroll
  for (int i = 0; i < 4; ++i) m4[i] = m4[i] * d4[i] + hs * r4[i];
  st4(out, m4);
}

// Ht on nodes k0..k0+N-1 of edge e: d/dt Ht = (grad_s Er - (1/r) d(m Et)/dr)/mu0
// with odd (PEC) Et ghosts (solver.py:877-899, 443-456):
//   Ht += (Er_head - Er_tail) / theta_e * hA[k] - Et[k] * hU[k] + Et[k-1] * hD[k]
// (hA = dt/(mu0 r), hU / hD the upper / lower PEC-ghosted radial difference
// weights; y holds them for the run's nodes).  The run holding node 0 also
// advances the surface-impedance ADE
// (surface_impedance.py:225-270) from the edge's pole memory si_in (T reals,
// shared or global) into si_out (global) with the edge's scale *si_sp, unless
// hnew points at the node-0 value a separate pass already advanced.
// inv_t = 1 / primal edge angle.
// Per-layer factors of an edge's H run at nodes k0..k0+N-1: hA, hU, hD and
// whether midpoint k0 exists (the run's upper Et).
template <typename real>
struct HEdgeLayer {
  Run<real> fa, fu, fd;
  bool up;
};
template <typename real>
__device__ __forceinline__ HEdgeLayer<real> h_edge_layer(const Rec<real>& R, const Layers<real>& Ls, int k0) {
  HEdgeLayer<real> y;
  y.fa = ld16(Ls.hA + k0);
  y.fu = ld16(Ls.hU + k0);
  y.fd = ld16(Ls.hD + k0);
  y.up = k0 < R.Pm;
  return y;
}

// The run's new values (h_edge_run stores them to htout).
template <typename real>
__device__ __forceinline__ Run<real> h_edge_value(const Rec<real>& R, const Layers<real>& Ls, const HEdgeLayer<real>& y,
                                                  int e, int k0, const real* erh, const real* ert, const real* etr,
                                                  const real* hto, real inv_t, const real* si_in, real* si_out,
                                                  const real* si_sp, const real* hnew) {
  constexpr int N = Lanes<real>::N;
  const Run<real> vh = ld16(erh + k0), vt = ld16(ert + k0), vo = ld16(hto + k0);
  const Run<real> vu = y.up ? ld16(etr + k0) : zero_run<real>();
  const real vprev = k0 > 0 ? etr[k0 - 1] : real(0);
  const Run<real>&fa = y.fa, &fu = y.fu, &fd = y.fd;
  Run<real> out;
#pragma unroll
  for (int r = 0; r < N; ++r) {
    const real dn = r == 0 ? vprev : vu.x[r - 1];
    out.x[r] = vo.x[r] + ((vh.x[r] - vt.x[r]) * inv_t) * fa.x[r] - vu.x[r] * fu.x[r] + dn * fd.x[r];
  }
  if (R.si_terms > 0 && k0 == 0) {
    if (hnew) {
      out.x[0] = *hnew;  // advanced by the patch's surface-impedance pass
    } else {
      const int T = R.si_terms;
      const real h_old = vo.x[0];
      const real g0 = (vh.x[0] - vt.x[0]) * inv_t * Ls.invr[0];
      const real e1 = R.si_metric * vu.x[0];
      const real s = *si_sp;
      const real h_new = si_boundary(R, h_old, g0, e1, s, si_history(si_in, Ls.si_hist, T));
      const real hs = h_new + h_old;
      if ((T & 3) == 0) {
        for (int p = 0; p < T; p += 4) si_update_quad(si_in + p, si_out + p, Ls, p, hs);
      } else {
        for (int p = 0; p < T; ++p) si_out[p] = si_in[p] * Ls.si_decay[p] + hs * Ls.si_drive[p];
      }
      out.x[0] = h_new;
    }
  }
  return out;
}

template <typename real>
__device__ __forceinline__ void h_edge_run(const Rec<real>& R, const Layers<real>& Ls, const HEdgeLayer<real>& y, int e,
                                           int k0, const real* erh, const real* ert, const real* etr, const real* hto,
                                           real* htout, real inv_t, const real* si_in, real* si_out, const real* si_sp,
                                           const real* hnew = nullptr) {
  st16(htout + k0, h_edge_value(R, Ls, y, e, k0, erh, ert, etr, hto, inv_t, si_in, si_out, si_sp, hnew));
}

// New Hr at one face run from the old run hv, the three edges' Et runs and the
// face's circulation weights w0..w2 (fc = hC at the run's midpoints).
template <typename real>
__device__ __forceinline__ Run<real> hr_value(const Run<real>& hv, const Run<real>& a0, const Run<real>& a1,
                                              const Run<real>& a2, real w0, real w1, real w2, const Run<real>& fc) {
  Run<real> hn;
#pragma unroll
  for (int r = 0; r < Lanes<real>::N; ++r) hn.x[r] = hv.x[r] - (w0 * a0.x[r] + w1 * a1.x[r] + w2 * a2.x[r]) * fc.x[r];
  return hn;
}

// Hr and the plasma current on midpoints j0..j0+N-1 of face f
// (solver.py:915-921; plasma.py:413-442, 489-501):
//   Hr -= (sum_i sign_i theta_i Et_i / A_f) * hC[j],  hC = dt / (mu0 m).
// The face's (3, Pm) input current rows of species s are at jin0 + s *
// jin_stride (jin0 == nullptr: the state arrays R.J[s] themselves); outputs go
// to R.J[s].  fw is the face's circulation row (4 reals) and gp its
// reconstruction row (12 reals); fc is hC at the run's midpoints.
template <typename real, bool PLASMA>
__device__ __forceinline__ void h_face_run(const Rec<real>& R, const Layers<real>& Ls, const Run<real>& fc, int f,
                                           int j0, const real* et0, const real* et1, const real* et2, const real* hro,
                                           real* hrout, const real* pa, const real* pb, const real* pc,
                                           const real* jin0, int jin_stride, real* jtot, const real* fw,
                                           const real* gp) {
  constexpr int N = Lanes<real>::N;
  const int L = R.L, Pn = R.Pn, Pm = R.Pm;
  const Run<real> a0 = ld16(et0 + j0), a1 = ld16(et1 + j0), a2 = ld16(et2 + j0);
  const Run<real> hv = ld16(hro + j0);
  real wv[4];
  ld4(fw, wv);
  const real w0 = wv[0], w1 = wv[1], w2 = wv[2];
  st16(hrout + j0, hr_value(hv, a0, a1, a2, w0, w1, w2, fc));
  if (!PLASMA) return;
  // radial E at midpoints: mean of the three vertices' nodes j and j+1
  const Run<real> na = ld16(pa + j0), nb = ld16(pb + j0), nc = ld16(pc + j0);
  const bool more = j0 + N < Pn;
  const real ta = more ? pa[j0 + N] : real(0), tb = more ? pb[j0 + N] : real(0), tc = more ? pc[j0 + N] : real(0);
  real sum[N + 1];
#pragma unroll
  for (int r = 0; r < N; ++r) sum[r] = na.x[r] + nb.x[r] + nc.x[r];
  sum[N] = ta + tb + tc;
  real rc[3][3], cf[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    real g[4];
    ld4(gp + 4 * i, g);
#pragma unroll
    for (int c = 0; c < 3; ++c) rc[i][c] = g[c];
    cf[i] = g[3];
  }
  const real sixth = real(1) / real(6);
  real E[N][3];
#pragma unroll
  for (int r = 0; r < N; ++r) {
    const real rad = (sum[r] + sum[r + 1]) * sixth;
#pragma unroll
    for (int c = 0; c < 3; ++c) E[r][c] = a0.x[r] * rc[0][c] + a1.x[r] * rc[1][c] + a2.x[r] * rc[2][c] + rad * cf[c];
  }
  real tot[N][3];
#pragma unroll
  for (int r = 0; r < N; ++r) tot[r][0] = tot[r][1] = tot[r][2] = real(0);
  const bool tail = j0 + N > L;  // the run holds padding midpoints
  const bool full_rows = R.plasma_full != 0, mag = R.magnetized != 0;
  for (int s = 0; s < R.n_species; ++s) {
    real* jo = R.J[s] + (size_t)f * 3 * Pm;
    const real* ji = jin0 ? jin0 + (size_t)s * jin_stride : jo;
    Run<real> jc[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) jc[c] = ld16(ji + c * Pm + j0);
    // coefficient rows of species s: decay, cos, sin, parallel drive, drive, cross drive
    auto crow = [&](int c) -> Run<real> {
      return full_rows ? ldg16(R.pcoef + ((size_t)(s * 6 + c) * R.nF + f) * Pm + j0) : ld16(Ls.pc + (s * 6 + c) * Pm + j0);
    };
    const Run<real> decay = crow(0), dre = crow(4);
    Run<real> jn[3];
    if (mag) {
      const Run<real> cs = crow(1), sn = crow(2), dpar = crow(3), dim = crow(5);
      Run<real> bd[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) bd[c] = full_rows ? ldg16(R.bdir + ((size_t)f * 3 + c) * Pm + j0) : ld16(Ls.bd + c * Pm + j0);
#pragma unroll
      for (int r = 0; r < N; ++r) {
        const real b[3] = {bd[0].x[r], bd[1].x[r], bd[2].x[r]};
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
        const real J0 = jc[0].x[r], J1 = jc[1].x[r], J2 = jc[2].x[r];
        const real jb = J0 * b[0] + J1 * b[1] + J2 * b[2];
        real Jp[3], Jq[3], Jx[3];
        Jp[0] = jb * b[0];
        Jp[1] = jb * b[1];
        Jp[2] = jb * b[2];
        Jq[0] = J0 - Jp[0];
        Jq[1] = J1 - Jp[1];
        Jq[2] = J2 - Jp[2];
        Jx[0] = Jq[1] * b[2] - Jq[2] * b[1];
        Jx[1] = Jq[2] * b[0] - Jq[0] * b[2];
        Jx[2] = Jq[0] * b[1] - Jq[1] * b[0];
#pragma unroll
        for (int c = 0; c < 3; ++c)
          jn[c].x[r] = decay.x[r] * Jp[c] + dpar.x[r] * Ep[c] + decay.x[r] * (cs.x[r] * Jq[c] + sn.x[r] * Jx[c]) +
                       dre.x[r] * Eq[c] + dim.x[r] * Ex[c];
      }
    } else {
      // B = 0 everywhere: the rotation angle is 0 and its cosine exactly 1, so
      // decay * (cos * J) is decay * J bit for bit (plasma.py:430-439)
#pragma unroll
      for (int r = 0; r < N; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) jn[c].x[r] = decay.x[r] * jc[c].x[r] + dre.x[r] * E[r][c];
    }
    if (tail) {
#pragma unroll
      for (int r = 0; r < N; ++r)
        if (j0 + r >= L) jn[0].x[r] = jn[1].x[r] = jn[2].x[r] = real(0);
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
#pragma unroll
      for (int r = 0; r < N; ++r) tot[r][c] += jn[c].x[r];
      st16(jo + c * Pm + j0, jn[c]);
    }
  }
  if (R.n_species > 1) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      Run<real> t;
#pragma unroll
      for (int r = 0; r < N; ++r) t.x[r] = tot[r][c];
      st16(jtot + c * Pm + j0, t);
    }
  }
}

// Per-layer factors of a vertex run at nodes k0..k0+N-1: 1/r, the loss
// coefficients (shared rows, or vertex v's own rows when the material varies
// horizontally), the node weights of the midpoints below / above, and whether
// midpoints k0-1 (below) and k0 (in) exist.
template <typename real>
struct VertexLayer {
  Run<real> ir, ca, cb, wl, wu;
  bool in, below;
};
template <typename real>
__device__ __forceinline__ VertexLayer<real> vertex_layer(const Rec<real>& R, const Layers<real>& Ls, int v, int k0) {
  VertexLayer<real> y;
  y.ir = ld16(Ls.invr + k0);
  y.ca = R.coef_full ? ldg16(R.ca_er + (size_t)v * R.Pn + k0) : ld16(Ls.ca_er + k0);
  y.cb = R.coef_full ? ldg16(R.cb_er + (size_t)v * R.Pn + k0) : ld16(Ls.cb_er + k0);
  y.wl = ld16(Ls.vwl + k0);
  y.wu = ld16(Ls.vwu + k0);
  y.in = k0 < R.Pm;
  y.below = k0 >= 1 && k0 - 1 < R.L;
  return y;
}

// Per-layer factors of an edge run at midpoints j0..j0+N-1: 1/m, the radial
// curl weights, the loss coefficients (shared rows or edge e's own rows) and
// whether node j0+N exists.
template <typename real>
struct EdgeLayer {
  Run<real> im, fu, fd, ca, cb;
  bool tail;
};
template <typename real>
__device__ __forceinline__ EdgeLayer<real> edge_layer(const Rec<real>& R, const Layers<real>& Ls, int e, int j0) {
  EdgeLayer<real> y;
  y.im = ld16(Ls.invm + j0);
  y.fu = ld16(Ls.eU + j0);
  y.fd = ld16(Ls.eD + j0);
  y.ca = R.coef_full ? ldg16(R.ca_et + (size_t)e * R.Pm + j0) : ld16(Ls.ca_et + j0);
  y.cb = R.coef_full ? ldg16(R.cb_et + (size_t)e * R.Pm + j0) : ld16(Ls.cb_et + j0);
  y.tail = j0 + Lanes<real>::N < R.Pn;
  return y;
}

// Er on nodes k0..k0+N-1 of vertex v (solver.py:929-962; plasma.py:511-526):
//   Er = Ca Er + Cb (circ_v(Ht) / r - J_r) - source,
// J_r the vertex's area-averaged radial current at the node (weights vwl / vwu
// of the midpoints below / above).  y: the run's layer factors; src: whether v
// may carry a vertical source support (else the source list is not searched).
// hrows[q]: Ht row of slot q's edge; jrows[q]: (3, Pm) summed current rows of
// slot q's face; coef[q] = sign * phi_e / A*_v and wcs[4q..4q+2] = area weight
// * face centre of slot q (zero in padding slots).  rav_in: the vertex's
// radial current at midpoints k0-1 .. k0+N-1 (N+1 values, zero where a
// midpoint does not exist), computed by the caller with rav_term in slot order
// (the same bits as accumulating it here), or nullptr to accumulate it here.
template <typename real, bool PLASMA, int MAXDEG>
__device__ __forceinline__ void e_vertex_run(const Rec<real>& R, const VertexLayer<real>& y, bool src, int v, int k0,
                                             const real* const* hrows, const real* const* jrows, const real* coef,
                                             const real* wcs, const real* ero, real* erout, real current,
                                             const real* rav_in = nullptr) {
  constexpr int N = Lanes<real>::N;
  const int Pm = R.Pm;
  Run<real> hv[MAXDEG];
#pragma unroll
  for (int q = 0; q < MAXDEG; ++q) hv[q] = ld16(hrows[q] + k0);
  const Run<real> ev = ld16(ero + k0);
  const Run<real>&ir = y.ir, &ca = y.ca, &cb = y.cb;
  real cq[(MAXDEG + 3) / 4 * 4];
#pragma unroll
  for (int q = 0; q < MAXDEG; q += 4) {
    real c4[4];
    ld4(coef + q, c4);
#pragma unroll
    for (int i = 0; i < 4; ++i) cq[q + i] = c4[i];
  }
  real acc[N];
#pragma unroll
  for (int r = 0; r < N; ++r) {
    acc[r] = real(0);
#pragma unroll
    for (int q = 0; q < MAXDEG; ++q) acc[r] += cq[q] * hv[q].x[r];
  }
  Run<real> out;
#pragma unroll
  for (int r = 0; r < N; ++r) out.x[r] = ca.x[r] * ev.x[r] + cb.x[r] * (acc[r] * ir.x[r]);
  if (src && source_hit(R.src_er_v, R.n_src_er, v)) {
#pragma unroll
    for (int r = 0; r < N; ++r)
      for (int s = 0; s < R.n_src_er; ++s)
        if (R.src_er_v[s] == v && R.src_er_k[s] == k0 + r) out.x[r] -= R.src_er_c[s] * current;
  }
  if (PLASMA) {
    // radial current at faces (J . centre), area-averaged to the vertex, at
    // midpoints k0-1 .. k0+N-1
    real rav[N + 1];
#pragma unroll
    for (int r = 0; r <= N; ++r) rav[r] = real(0);
    const bool in = y.in, below = y.below;
    if (rav_in) {
#pragma unroll
      for (int r = 0; r <= N; ++r) rav[r] = rav_in[r];
    } else if (R.plasma_local) {
      real w[(MAXDEG + 3) / 4 * 4];
      slot_weights<real, MAXDEG>(wcs, w);
#pragma unroll
      for (int q = 0; q < MAXDEG; ++q) {
        const real* jf = jrows[q];
        const Run<real> jr = in ? ld16(jf + k0) : zero_run<real>();
        if (below) rav[0] = rav_local(rav[0], jf[k0 - 1], w[q]);
#pragma unroll
        for (int r = 0; r < N; ++r) rav[r + 1] = rav_local(rav[r + 1], jr.x[r], w[q]);
      }
    } else {
#pragma unroll
      for (int q = 0; q < MAXDEG; ++q) {
        real wc[4];
        ld4(wcs + 4 * q, wc);
        const real c0 = wc[0], c1 = wc[1], c2 = wc[2];
        const real* jf = jrows[q];
        const Run<real> jx = in ? ld16(jf + k0) : zero_run<real>();
        const Run<real> jy = in ? ld16(jf + Pm + k0) : zero_run<real>();
        const Run<real> jz = in ? ld16(jf + 2 * Pm + k0) : zero_run<real>();
        if (below) rav[0] = rav_term(rav[0], jf[k0 - 1], jf[Pm + k0 - 1], jf[2 * Pm + k0 - 1], c0, c1, c2);
#pragma unroll
        for (int r = 0; r < N; ++r) rav[r + 1] = rav_term(rav[r + 1], jx.x[r], jy.x[r], jz.x[r], c0, c1, c2);
      }
    }
#pragma unroll
    for (int r = 0; r < N; ++r) out.x[r] -= cb.x[r] * (y.wl.x[r] * rav[r] + y.wu.x[r] * rav[r + 1]);
  }
  st16(erout + k0, out);
}

// Et on midpoints j0..j0+N-1 of edge e (solver.py:964-989; plasma.py:503-509):
//   Et = Ca Et + Cb ((Hr_l - Hr_r) / phi_e / m - Ht[j+1] eU + Ht[j] eD - J_t) - source,
// eU / eD the radial curl weights of the nodes above / below, J_t the mean of
// the two faces' currents along the edge.  y: the run's layer factors; src:
// whether e may carry a tangential source support.  inv_p = 1 / dual edge
// angle; tp = left tangent, 0, right tangent, 0.
template <typename real, bool PLASMA>
__device__ __forceinline__ void e_edge_run(const Rec<real>& R, const EdgeLayer<real>& y, bool src, int e, int j0,
                                           const real* hl, const real* hq, const real* hto, const real* jl,
                                           const real* jq, const real* eto, real* etout, real current, real inv_p,
                                           const real* tp) {
  constexpr int N = Lanes<real>::N;
  const int Pm = R.Pm;
  const Run<real> a = ld16(hl + j0), b = ld16(hq + j0), hv = ld16(hto + j0), ev = ld16(eto + j0);
  const real htail = y.tail ? hto[j0 + N] : real(0);
  const Run<real>&im = y.im, &fu = y.fu, &fd = y.fd, &ca = y.ca, &cb = y.cb;
  Run<real> out;
#pragma unroll
  for (int r = 0; r < N; ++r) {
    const real hnext = (r + 1 < N) ? hv.x[r + 1] : htail;
    const real g = (a.x[r] - b.x[r]) * inv_p * im.x[r] - hnext * fu.x[r] + hv.x[r] * fd.x[r];
    out.x[r] = ca.x[r] * ev.x[r] + cb.x[r] * g;
  }
  if (src && source_hit(R.src_et_e, R.n_src_et, e)) {
#pragma unroll
    for (int r = 0; r < N; ++r)
      for (int s = 0; s < R.n_src_et; ++s)
        if (R.src_et_e[s] == e && R.src_et_j[s] == j0 + r) out.x[r] -= R.src_et_c[s] * current;
  }
  if (PLASMA && R.plasma_local) {
    // face frames: the edge tangents lie in the faces' tangent planes, so
    // only components 1 and 2 of each face's current enter; tp = left
    // tangent (1, 2), right tangent (1, 2)
    real t4[4];
    ld4(tp, t4);
    const Run<real> ly = ld16(jl + Pm + j0), lz = ld16(jl + 2 * Pm + j0);
    const Run<real> qy = ld16(jq + Pm + j0), qz = ld16(jq + 2 * Pm + j0);
#pragma unroll
    for (int r = 0; r < N; ++r) {
      const real left = ly.x[r] * t4[0] + lz.x[r] * t4[1];
      const real right = qy.x[r] * t4[2] + qz.x[r] * t4[3];
      out.x[r] -= cb.x[r] * (real(0.5) * (left + right));
    }
  } else if (PLASMA) {
    real tl[4], tq[4];
    ld4(tp, tl);
    ld4(tp + 4, tq);
    const real l0 = tl[0], l1 = tl[1], l2 = tl[2];
    const real q0 = tq[0], q1 = tq[1], q2 = tq[2];
    const Run<real> lx = ld16(jl + j0), ly = ld16(jl + Pm + j0), lz = ld16(jl + 2 * Pm + j0);
    const Run<real> qx = ld16(jq + j0), qy = ld16(jq + Pm + j0), qz = ld16(jq + 2 * Pm + j0);
#pragma unroll
    for (int r = 0; r < N; ++r) {
      const real left = lx.x[r] * l0 + ly.x[r] * l1 + lz.x[r] * l2;
      const real right = qx.x[r] * q0 + qy.x[r] * q1 + qz.x[r] * q2;
      out.x[r] -= cb.x[r] * (real(0.5) * (left + right));
    }
  }
  st16(etout + j0, out);
}

// ---------------------------------------------------------------------------
// Direct kernels: neighbour rows read straight from global memory (used when a
// patch's staged rows would not fit in shared memory).
// ---------------------------------------------------------------------------
template <typename real, bool PLASMA>
__global__ void __launch_bounds__(256) kh_kernel(const Rec<real>* __restrict__ recs, const int2* __restrict__ block_map,
                                                  int n_members) {
  constexpr int N = Lanes<real>::N;
  extern __shared__ __align__(16) unsigned char dyn_smem[];
  __shared__ Rec<real> R;
  int member, patch;
  member_patch(block_map, n_members, member, patch);
  load_rec(R, recs + member);
  Layers<real> Ls;
  load_layers(R, reinterpret_cast<real*>(dyn_smem), Ls);
  const int Pn = R.Pn, Pm = R.Pm, cn = Pn / N, cm = Pm / N;
  const uint32_t mag_cn = div_magic(cn), mag_cm = div_magic(cm);
  const int ea = R.eptr_h[patch], eb = R.eptr_h[patch + 1];
  for (int it = threadIdx.x; it < (eb - ea) * cn; it += blockDim.x) {
    const int el = fast_div(it, mag_cn);
    const int e = ea + el;
    const int2 th = __ldg(R.edge_th + e);
    const int k0 = (it - el * cn) * N;
    h_edge_run(R, Ls, h_edge_layer(R, Ls, k0), e, k0, R.er + (size_t)th.y * Pn, R.er + (size_t)th.x * Pn, R.et + (size_t)e * Pm,
               R.ht + (size_t)e * Pn, R.ht + (size_t)e * Pn, __ldg(R.inv_theta + e), R.si_mem + (size_t)e * R.si_terms,
               R.si_mem + (size_t)e * R.si_terms, R.si_scale + e);
  }
  const int fa = patch * R.fpp_h, fb = min(fa + R.fpp_h, R.nF);
  for (int it = threadIdx.x; it < (fb - fa) * cm; it += blockDim.x) {
    const int fl = fast_div(it, mag_cm);
    const int f = fa + fl;
    const int4 fe = __ldg(R.face_e + f);
    const int4 fv = PLASMA ? __ldg(R.face_v + f) : make_int4(0, 0, 0, 0);
    const int j0 = (it - fl * cm) * N;
    h_face_run<real, PLASMA>(R, Ls, ld16(Ls.hC + j0), f, j0, R.et + (size_t)fe.x * Pm, R.et + (size_t)fe.y * Pm,
                             R.et + (size_t)fe.z * Pm, R.hr + (size_t)f * Pm, R.hr + (size_t)f * Pm,
                             R.er + (size_t)fv.x * Pn, R.er + (size_t)fv.y * Pn, R.er + (size_t)fv.z * Pn, nullptr, 0,
                             R.n_species > 1 ? R.Jtot + (size_t)f * 3 * Pm : nullptr, R.face_w + 4 * (size_t)f,
                             PLASMA ? R.face_pl + 12 * (size_t)f : nullptr);
  }
}

template <typename real, bool PLASMA, int MAXDEG>
__global__ void __launch_bounds__(256) ke_kernel(const Rec<real>* __restrict__ recs, const int2* __restrict__ block_map,
                                                  int n_members, int istep) {
  constexpr int N = Lanes<real>::N;
  extern __shared__ __align__(16) unsigned char dyn_smem[];
  __shared__ Rec<real> R;
  int member, patch;
  member_patch(block_map, n_members, member, patch);
  load_rec(R, recs + member);
  Layers<real> Ls;
  load_layers(R, reinterpret_cast<real*>(dyn_smem), Ls);
  const int Pn = R.Pn, Pm = R.Pm, SW = R.slot_width, cn = Pn / N, cm = Pm / N;
  const uint32_t mag_cn = div_magic(cn), mag_cm = div_magic(cm);
  const real current = (R.n_src_er + R.n_src_et) > 0 ? (real)R.cur[istep] : real(0);
  const real* Jsum = PLASMA ? jsum(R) : nullptr;
  const int va = R.vptr[patch], vb = R.vptr[patch + 1];
  for (int it = threadIdx.x; it < (vb - va) * cn; it += blockDim.x) {
    const int vl = fast_div(it, mag_cn);
    const int slot = va + vl;
    const int v = __ldg(R.vlist + slot);
    const real* hrows[MAXDEG];
    const real* jrows[MAXDEG];
#pragma unroll
    for (int q = 0; q < MAXDEG; ++q) {
      hrows[q] = R.ht + (size_t)__ldg(R.ps_edge + (size_t)slot * SW + q) * Pn;
      jrows[q] = PLASMA ? Jsum + (size_t)__ldg(R.ps_face + (size_t)slot * SW + q) * 3 * Pm : nullptr;
    }
    const int k0 = (it - vl * cn) * N;
    e_vertex_run<real, PLASMA, MAXDEG>(R, vertex_layer(R, Ls, v, k0), R.n_src_er > 0, v, k0, hrows, jrows,
                                       R.ps_coef + (size_t)slot * SW,
                                       PLASMA ? R.ps_wc + (size_t)slot * SW * 4 : nullptr, R.er + (size_t)v * Pn,
                                       R.er + (size_t)v * Pn, current);
  }
  const int ea = R.eptr_e[patch], eb = R.eptr_e[patch + 1];
  for (int it = threadIdx.x; it < (eb - ea) * cm; it += blockDim.x) {
    const int el = fast_div(it, mag_cm);
    const int e = ea + el;
    const int2 lr = __ldg(R.edge_lr + e);
    const int j0 = (it - el * cm) * N;
    e_edge_run<real, PLASMA>(R, edge_layer(R, Ls, e, j0), R.n_src_et > 0, e, j0, R.hr + (size_t)lr.x * Pm,
                             R.hr + (size_t)lr.y * Pm,
                             R.ht + (size_t)e * Pn, PLASMA ? Jsum + (size_t)lr.x * 3 * Pm : nullptr,
                             PLASMA ? Jsum + (size_t)lr.y * 3 * Pm : nullptr, R.et + (size_t)e * Pm,
                             R.et + (size_t)e * Pm, current, __ldg(R.inv_phi + e), PLASMA ? R.tan + 8 * (size_t)e : nullptr);
  }
}

// ---------------------------------------------------------------------------
// Plasma current between the Cartesian frame of the caller's state and the
// face frames the step kernels read when Rec::plasma_local is set: rows of Q
// (F, 12) are e0 (along the face centre), e1, e2, each padded to four reals.
// to_local: J <- Q J; else J <- Q^T J, midpoint quad by midpoint quad of one
// species' (F, 3, Pm) buffer.  Zero padding midpoints stay zero.
// ---------------------------------------------------------------------------
template <typename real>
__global__ void __launch_bounds__(256) plasma_frame_kernel(real* __restrict__ J, const real* __restrict__ Q, int nF,
                                                           int Pm, int to_local) {
  constexpr int N = Lanes<real>::N;
  const int cm = Pm / N;
  const long long n = (long long)nF * cm;
  for (long long it = blockIdx.x * (long long)blockDim.x + threadIdx.x; it < n;
       it += (long long)gridDim.x * blockDim.x) {
    const int f = (int)(it / cm);
    const int j0 = (int)(it - (long long)f * cm) * N;
    real q[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int c = 0; c < 3; ++c) q[i][c] = __ldg(Q + 12 * (size_t)f + 4 * i + c);
    real* base = J + (size_t)f * 3 * Pm + j0;
    const Run<real> a = ld16(base), b = ld16(base + Pm), c = ld16(base + 2 * Pm);
    Run<real> o[3];
#pragma unroll
    for (int r = 0; r < N; ++r)
#pragma unroll
      for (int i = 0; i < 3; ++i)
        o[i].x[r] = to_local ? q[i][0] * a.x[r] + q[i][1] * b.x[r] + q[i][2] * c.x[r]
                             : q[0][i] * a.x[r] + q[1][i] * b.x[r] + q[2][i] * c.x[r];
    st16(base, o[0]);
    st16(base + Pm, o[1]);
    st16(base + 2 * Pm, o[2]);
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
  const int pitch = (kind == 0 || kind == 3) ? rec->Pn : rec->Pm;
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

// One member's probe in a batched sampling launch: the member's record,
// field kind, rows, support width, the probe's device tables and the row of
// its staging buffer that this step writes.
struct ProbeRef {
  int member, kind, rows, width;
  const int* index;
  const int* layer;
  const double* weight;
  double* staging;  // column 0 of this probe's rows in the (chunk, total rows) staging
};

// Receiver rows of every member of an ensemble in one launch: warp w samples
// global row w; rowmap[w] = {probe, row within that probe}.  Same arithmetic
// as sample_rec_kernel; step `step_row` of the chunk goes to row step_row of
// the (chunk, total_rows) staging.
template <typename real>
__global__ void sample_batch_kernel(const Rec<real>* __restrict__ recs, const ProbeRef* __restrict__ refs,
                                    const int2* __restrict__ rowmap, int total_rows, int step_row) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= total_rows) return;
  const int2 rm = rowmap[warp];
  const ProbeRef pr = refs[rm.x];
  const Rec<real>* rec = recs + pr.member;
  const real* field = pr.kind == 0 ? rec->er : pr.kind == 1 ? rec->et : pr.kind == 2 ? rec->hr : rec->ht;
  const int pitch = (pr.kind == 0 || pr.kind == 3) ? rec->Pn : rec->Pm;
  double acc = 0.0;
  for (int q = lane; q < pr.width; q += 32) {
    const int o = rm.y * pr.width + q;
    acc += pr.weight[o] * (double)field[(size_t)pr.index[o] * pitch + pr.layer[o]];
  }
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) acc += __shfl_down_sync(0xFFFFFFFFu, acc, s);
  if (lane == 0) pr.staging[(size_t)step_row * total_rows + rm.y] = acc;
}

// max |x| of up to four arrays; results combined with an order-independent
// atomic max on the bit pattern of non-negative doubles (NaN sorts above +Inf,
// so a non-finite field reports NaN or Inf).  Row padding is zero and does not
// change a maximum of absolute values.
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
