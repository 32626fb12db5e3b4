// C ABI of the geodesic FDTD engine: plan construction, the step loop (direct
// launches or CUDA-graph chunks), observation probes, reductions and the
// ArrayBackend primitives.  Declarations and reference citations: include/ifdtd.h.
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/ifdtd.h"
#include "errors.cuh"
#include "fused_kernels.cuh"
#include "pipe_kernels.cuh"
#include "step_kernels.cuh"

using namespace ifdtd;

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

}  // namespace

int ifdtd::record_error(int code, const std::string& msg) { return fail(code, msg); }

namespace {

#define CUDA_TRY(expr)                                                                          \
  do {                                                                                          \
    cudaError_t _e = (expr);                                                                    \
    if (_e != cudaSuccess)                                                                      \
      return fail(IFDTD_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(_e));          \
  } while (0)

struct DeviceArena {
  std::vector<void*> blocks;
  size_t bytes = 0;
  ~DeviceArena() {
    for (void* p : blocks) cudaFree(p);
  }
  template <typename T>
  cudaError_t upload(const std::vector<T>& host, const T** out) {
    *out = nullptr;
    if (host.empty()) return cudaSuccess;
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, host.size() * sizeof(T));
    if (e != cudaSuccess) return e;
    blocks.push_back(p);
    bytes += host.size() * sizeof(T);
    e = cudaMemcpy(p, host.data(), host.size() * sizeof(T), cudaMemcpyHostToDevice);
    *out = static_cast<const T*>(p);
    return e;
  }
  cudaError_t alloc(size_t n, void** out) {
    *out = nullptr;
    if (n == 0) return cudaSuccess;
    cudaError_t e = cudaMalloc(out, n);
    if (e != cudaSuccess) return e;
    blocks.push_back(*out);
    bytes += n;
    return cudaSuccess;
  }
};

}  // namespace

struct ifdtd_probe {
  ifdtd_plan* plan;
  int kind, rows, width;
  int* index = nullptr;
  int* layer = nullptr;
  double* weight = nullptr;
  double* staging = nullptr;  // (graph_chunk, rows)
  DeviceArena arena;          // the probe's own device buffers
};

struct GraphEntry {
  int chunk;
  const ifdtd_probe* probe;
  cudaGraphExec_t exec;
};

struct ifdtd_plan {
  int dtype = 4;
  int device = 0;
  int nV = 0, nE = 0, nF = 0, L = 0, T = 0, S = 0;
  int n_patches = 0, n_patches_e = 0, threads = 256, chunk = 32, maxdeg = 6, Pn = 0, Pm = 0;
  int h_mode = 1, e_mode = 1;  // 1 direct gathers, 2 pipeline
  int pipe_copy = 0;           // pipeline copy engine: 0 TMA bulk copies, 1 cp.async
  int producers = 2;           // copy-issuing warps per pipelined CTA
  int lanes = 0;               // lane layout of the pipelined consumers: 0 packed rows, 1 rows on 8-lane boundaries
  int e_threads = 0;           // compute threads of a pipelined E-phase CTA (above 384 - 32 x e_producers: wide CTAs)
  int e_producers = 2;         // copy-issuing warps of a pipelined E-phase CTA
  bool pipe_h_ok = false, pipe_e_ok = false;
  int kh_stage = 0, ke_stage = 0, kh_stages = 0, ke_stages = 0, kh_grid = 0, ke_grid = 0, sm_count = 148;
  size_t smem_bytes = 0, kh_smem = 0, ke_smem = 0;
  int* d_status = nullptr;
  bool plasma = false;
  bool plasma_local = false;     // the plasma current runs in face frames (converted around every call)
  const void* d_frame = nullptr;  // (F, 12) face-frame rows of those conversions
  DeviceArena arena;
  void* d_rec = nullptr;               // Rec<real> in device memory
  std::vector<unsigned char> h_rec;    // host image of the record
  double* d_cur = nullptr;             // staging currents (chunk)
  void* d_jtot = nullptr;              // summed species current (S > 1)
  // primitive tables
  const int2* edge_th = nullptr;
  const int2* edge_lr = nullptr;
  const int4* face_e = nullptr;
  const int* face_sign = nullptr;
  const int* v_off = nullptr;
  const int* v_edge = nullptr;
  const int* v_sign = nullptr;
  ifdtd_state last_state;
  bool have_state = false;
  cudaStream_t capture_stream = nullptr;
  std::vector<GraphEntry> graphs;
  std::vector<ifdtd_probe*> probes;
  std::vector<float> kh_cost, ke_cost;  // staged bytes per pipelined patch (balances batched launches)
  // fused step: halo tables, the record of the second field copy and its arrays
  bool fused = false;
  bool fused_pipe = false;  // the fused step through the ring (pipe::kf_tma) rather than direct gathers
  int kf_stage = 0, kf_stages = 0, kf_grid = 0, kf_threads = 0, kf_producers = 0, kf_lanes = 0;
  size_t kf_smem = 0;
  std::vector<float> kf_cost;  // staged bytes per fused patch (balances batched launches)
  FusedTables fused_tab{};
  size_t fused_smem = 0;
  void* d_rec_b = nullptr;
  void* fb[4] = {nullptr, nullptr, nullptr, nullptr};  // second er, et, hr, ht
  size_t fb_bytes[4] = {0, 0, 0, 0};
  ~ifdtd_plan() {
    for (auto& g : graphs) cudaGraphExecDestroy(g.exec);
    if (capture_stream) cudaStreamDestroy(capture_stream);
  }
};

namespace {

template <typename real>
std::vector<real> cast(const double* p, size_t n) {
  std::vector<real> out(n);
  for (size_t i = 0; i < n; ++i) out[i] = (real)p[i];
  return out;
}

bool in_range(const int64_t* p, size_t n, int64_t hi) {
  for (size_t i = 0; i < n; ++i)
    if (p[i] < 0 || p[i] >= hi) return false;
  return true;
}

int round4(int n) { return (n + 3) / 4 * 4; }

// ---------------------------------------------------------------------------
// Pipelined kernels: per patch, the rows it reads as copy descriptors (runs of
// consecutive rows of one source array) and a table blob whose local indices
// address the rows inside the patch's shared-memory stage.  Stage layout:
// [blob][gathered rows ...][own contiguous rows ...], every part 16-byte
// aligned (rows are padded to 16-byte pitches).
// ---------------------------------------------------------------------------
constexpr int kSmemPerBlock = 232448;  // opt-in dynamic shared memory per CTA on sm_100

struct PipeTables {
  std::vector<int> dptr{0};
  std::vector<int4> desc;
  std::vector<unsigned char> tab;
  int stage_bytes = 0;
};

// Sorted unique ids -> runs of consecutive rows, bridging gaps of at most
// `gap` rows; loc[id] = the id's position among the staged rows.  Returns the
// number of staged rows.
int make_runs(const std::vector<int>& ids, int gap, std::vector<std::pair<int, int>>& runs, std::vector<int>& loc) {
  runs.clear();
  int before = 0;
  for (const int id : ids) {
    if (!runs.empty() && id - (runs.back().first + runs.back().second) <= gap) {
      runs.back().second = id - runs.back().first + 1;
    } else {
      if (!runs.empty()) before += runs.back().second;
      runs.push_back({id, 1});
    }
    loc[id] = before + (id - runs.back().first);
  }
  return runs.empty() ? 0 : before + runs.back().second;
}

void sort_unique(std::vector<int>& v) {
  std::sort(v.begin(), v.end());
  v.erase(std::unique(v.begin(), v.end()), v.end());
}

// Append bytes to the blob (16-byte padded); returns the offset from `base`.
int blob_put(std::vector<unsigned char>& tab, size_t base, const void* src, size_t bytes) {
  const int off = (int)(tab.size() - base);
  const unsigned char* p = static_cast<const unsigned char*>(src);
  tab.insert(tab.end(), p, p + bytes);
  tab.resize((tab.size() + 15) / 16 * 16, 0);
  return off;
}

void add_runs(std::vector<int4>& desc, int src, const std::vector<std::pair<int, int>>& runs, int dst, int row_bytes) {
  int pos = 0;
  for (const auto& r : runs) {
    desc.push_back(make_int4(src, r.first, dst + pos * row_bytes, r.second * row_bytes));
    pos += r.second;
  }
}

int round128(int n) { return (n + 127) / 128 * 128; }

// Check every copy descriptor before upload: a positive multiple of 16 bytes
// of whole rows, a 16-byte aligned destination inside the patch's stage, source
// rows inside their array, the blob first and inside the table, and at most
// 2^20 - 1 bytes per patch (the mbarrier transaction limit).
bool descriptors_valid(const PipeTables& T, int rb, int Pn, int Pm, int Tsi, int nV, int nE, int nF, int S) {
  using namespace pipe;
  for (size_t q = 0; q + 1 < T.dptr.size(); ++q) {
    long total = 0;
    for (int d = T.dptr[q]; d < T.dptr[q + 1]; ++d) {
      const int4 x = T.desc[d];
      int row = 0;
      long rows = 0;
      switch (x.x) {
        case kSrcEr: row = Pn * rb; rows = nV; break;
        case kSrcEt: row = Pm * rb; rows = nE; break;
        case kSrcHt: row = Pn * rb; rows = nE; break;
        case kSrcHr: row = Pm * rb; rows = nF; break;
        case kSrcJsum: row = 3 * Pm * rb; rows = S > 0 ? nF : 0; break;
        case kSrcSi: row = Tsi * rb; rows = Tsi > 0 ? nE : 0; break;
        case kSrcTab: row = 16; rows = (long)(T.tab.size() / 16); break;
        default:
          if (x.x < kSrcJ0 || x.x >= kSrcJ0 + S) return false;
          row = 3 * Pm * rb;
          rows = nF;
      }
      if (row <= 0 || x.w <= 0 || x.w % 16 || x.w % row || x.z % 16 || x.z < 0 || x.z + x.w > T.stage_bytes) return false;
      if (x.y < 0 || (long)x.y + x.w / row > rows) return false;
      if ((x.x == kSrcTab) != (d == T.dptr[q]) || (x.x == kSrcTab && x.z != 0)) return false;
      total += x.w;
    }
    if (total >= (1 << 20)) return false;
  }
  return true;
}

// H phase (patch = faces [q*fpp, ...) and edges eptr[q]..eptr[q+1]).  Stage:
// blob, er rows (edge ends and, with plasma, face vertices), et rows (face
// edges, which include the owned edges), own ht rows, own hr rows, own
// current rows per species, own surface-impedance pole rows (Tsi reals each).
template <typename real>
bool build_pipe_h(PipeTables& T, int n, int fpp, int nF, const std::vector<int>& eptr, const std::vector<int2>& th,
                  const std::vector<int4>& fe, const std::vector<int4>& fv, const std::vector<real>& inv_theta,
                  const std::vector<real>& fw, const std::vector<real>& pl, int S, int Pn, int Pm, int Tsi,
                  const double* si_scale, std::vector<int>& locA, std::vector<int>& locB, int max_stage) {
  using namespace pipe;
  const int rb = (int)sizeof(real);
  if (Tsi > 0 && (Tsi * rb) % 16 != 0) return false;  // pole rows must be whole 16-byte units
  std::vector<real> sis;
  std::vector<int> er_ids, et_ids;
  std::vector<std::pair<int, int>> er_runs, et_runs;
  std::vector<int4> eloc, floc;
  for (int q = 0; q < n; ++q) {
    const int fa = q * fpp, fb = std::min(fa + fpp, nF), ea = eptr[q], eb = eptr[q + 1], ne = eb - ea, nf = fb - fa;
    er_ids.clear();
    et_ids.clear();
    for (int e = ea; e < eb; ++e) {
      er_ids.push_back(th[e].x);
      er_ids.push_back(th[e].y);
    }
    for (int f = fa; f < fb; ++f) {
      et_ids.push_back(fe[f].x);
      et_ids.push_back(fe[f].y);
      et_ids.push_back(fe[f].z);
      if (S > 0) {
        er_ids.push_back(fv[f].x);
        er_ids.push_back(fv[f].y);
        er_ids.push_back(fv[f].z);
      }
    }
    sort_unique(er_ids);
    sort_unique(et_ids);
    for (int e = ea; e < eb; ++e)
      if (!std::binary_search(et_ids.begin(), et_ids.end(), e)) return false;
    int gap = 0, n_er = 0, n_et = 0, nd = 0;
    for (;;) {
      n_er = make_runs(er_ids, gap, er_runs, locA);
      n_et = make_runs(et_ids, gap, et_runs, locB);
      nd = 1 + (int)er_runs.size() + (int)et_runs.size() + (ne > 0) + (nf > 0 ? 1 + S : 0) + (Tsi > 0 && ne > 0);
      if (nd <= kMaxDesc || gap >= 64) break;
      gap = 2 * gap + 1;
    }
    if (nd > kMaxDesc) return false;
    const size_t base = T.tab.size();
    int head[kh_head_ints] = {0};
    T.tab.resize(base + sizeof(head), 0);
    eloc.resize(ne);
    for (int el = 0; el < ne; ++el) {
      const int e = ea + el;
      eloc[el] = make_int4(locA[th[e].x], locA[th[e].y], locB[e], 0);
    }
    floc.resize(2 * (size_t)nf);
    for (int fl = 0; fl < nf; ++fl) {
      const int f = fa + fl;
      floc[2 * fl] = make_int4(locB[fe[f].x], locB[fe[f].y], locB[fe[f].z], S > 0 ? locA[fv[f].x] : 0);
      floc[2 * fl + 1] = make_int4(S > 0 ? locA[fv[f].y] : 0, S > 0 ? locA[fv[f].z] : 0, 0, 0);
    }
    head[kh_o_eloc] = blob_put(T.tab, base, eloc.data(), ne * sizeof(int4));
    head[kh_o_einv] = blob_put(T.tab, base, inv_theta.data() + ea, ne * (size_t)rb);
    head[kh_o_floc] = blob_put(T.tab, base, floc.data(), floc.size() * sizeof(int4));
    head[kh_o_fw] = blob_put(T.tab, base, fw.data() + 4 * (size_t)fa, 4 * (size_t)nf * rb);
    head[kh_o_fpl] = S > 0 ? blob_put(T.tab, base, pl.data() + 12 * (size_t)fa, 12 * (size_t)nf * rb) : head[kh_o_fw];
    if (Tsi > 0) {
      sis.resize(ne);
      for (int el = 0; el < ne; ++el) sis[el] = (real)si_scale[ea + el];
      head[kh_o_esis] = blob_put(T.tab, base, sis.data(), ne * (size_t)rb);
    } else {
      head[kh_o_esis] = head[kh_o_fw];
    }
    const int B = (int)(T.tab.size() - base);
    head[kh_ea] = ea;
    head[kh_ne] = ne;
    head[kh_fa] = fa;
    head[kh_nf] = nf;
    head[kh_o_er] = B;
    head[kh_o_et] = head[kh_o_er] + n_er * Pn * rb;
    head[kh_o_ht] = head[kh_o_et] + n_et * Pm * rb;
    head[kh_o_hr] = head[kh_o_ht] + ne * Pn * rb;
    head[kh_o_J] = head[kh_o_hr] + nf * Pm * rb;
    head[kh_o_si] = head[kh_o_J] + S * nf * 3 * Pm * rb;
    head[kh_o_hnew] = head[kh_o_si] + ne * Tsi * rb;  // scratch: node-0 Ht of the owned edges (not copied)
    const int end = head[kh_o_hnew] + (pipe::si_lane_groups(Tsi) ? (ne * rb + 15) / 16 * 16 : 0);
    if (round128(end) > max_stage) return false;  // the stage would not fit: stop early
    std::memcpy(T.tab.data() + base, head, sizeof(head));
    T.desc.push_back(make_int4(kSrcTab, (int)(base / 16), 0, B));
    add_runs(T.desc, kSrcEr, er_runs, head[kh_o_er], Pn * rb);
    add_runs(T.desc, kSrcEt, et_runs, head[kh_o_et], Pm * rb);
    if (ne > 0) T.desc.push_back(make_int4(kSrcHt, ea, head[kh_o_ht], ne * Pn * rb));
    if (nf > 0) {
      T.desc.push_back(make_int4(kSrcHr, fa, head[kh_o_hr], nf * Pm * rb));
      for (int s = 0; s < S; ++s)
        T.desc.push_back(make_int4(kSrcJ0 + s, fa, head[kh_o_J] + s * nf * 3 * Pm * rb, nf * 3 * Pm * rb));
    }
    if (Tsi > 0 && ne > 0) T.desc.push_back(make_int4(kSrcSi, ea, head[kh_o_si], ne * Tsi * rb));
    T.dptr.push_back((int)T.desc.size());
    T.stage_bytes = std::max(T.stage_bytes, round128(end));
    if (T.tab.size() / 16 >= (size_t)1 << 31) return false;
  }
  return true;
}

// E phase (patch = vertices vlist[vptr[q]..vptr[q+1]) and edges eptr[q]..).
// Stage: blob, ht rows (slot edges and owned edges), hr rows and summed
// current rows of one face set (faces beside owned edges and, with plasma,
// slot faces), own er rows (vertices in increasing order), own et rows.
template <typename real>
bool build_pipe_e(PipeTables& T, int n, const std::vector<int>& vptr, const std::vector<int>& vlist,
                  const std::vector<int>& eptr, const std::vector<int2>& lr, int SW, const std::vector<int>& ps_edge,
                  const std::vector<int>& ps_face, const std::vector<real>& ps_coef, const std::vector<real>& ps_wc,
                  const std::vector<real>& inv_phi, const std::vector<real>& tn, bool plasma, int Pn, int Pm,
                  const std::vector<char>& v_src, const std::vector<char>& e_src, std::vector<int>& locA,
                  std::vector<int>& locB, int max_stage, int min_gap) {
  using namespace pipe;
  const int rb = (int)sizeof(real);
  std::vector<int> h_ids, f_ids, v_ids, vloc;
  std::vector<std::pair<int, int>> h_runs, f_runs, v_runs;
  std::vector<std::pair<int, int>> own;  // (vertex, slot)
  std::vector<int> vid, vh, vj;
  std::vector<real> vcoef, vwc;
  std::vector<int4> eloc;
  vloc.assign(vlist.size(), 0);
  for (int q = 0; q < n; ++q) {
    const int va = vptr[q], vb = vptr[q + 1], ea = eptr[q], eb = eptr[q + 1], nv = vb - va, ne = eb - ea;
    own.clear();
    for (int sl = va; sl < vb; ++sl) own.push_back({vlist[sl], sl});
    std::sort(own.begin(), own.end());
    h_ids.clear();
    f_ids.clear();
    v_ids.clear();
    for (const auto& o : own) {
      v_ids.push_back(o.first);
      for (int k = 0; k < SW; ++k) {
        h_ids.push_back(ps_edge[(size_t)o.second * SW + k]);
        if (plasma) f_ids.push_back(ps_face[(size_t)o.second * SW + k]);
      }
    }
    for (int e = ea; e < eb; ++e) {
      h_ids.push_back(e);
      f_ids.push_back(lr[e].x);
      f_ids.push_back(lr[e].y);
    }
    sort_unique(h_ids);
    sort_unique(f_ids);
    make_runs(v_ids, 0, v_runs, vloc);
    // gaps of up to min_gap rows are always bridged (fewer, longer copies for
    // a few unread rows); wider ones only while the patch has too many copies
    int gap = min_gap, n_h = 0, n_f = 0, nd = 0;
    for (;;) {
      n_h = make_runs(h_ids, gap, h_runs, locA);
      n_f = make_runs(f_ids, gap, f_runs, locB);
      nd = 1 + (int)h_runs.size() + (int)f_runs.size() * (plasma ? 2 : 1) + (int)v_runs.size() + (ne > 0);
      if (nd <= kMaxDesc || gap >= 64) break;
      gap = 2 * gap + 1;
    }
    if (nd > kMaxDesc) return false;
    const size_t base = T.tab.size();
    int head[ke_head_ints] = {0};
    T.tab.resize(base + sizeof(head), 0);
    vid.assign(nv, 0);
    vh.assign((size_t)nv * SW, 0);
    vj.assign((size_t)nv * SW, 0);
    vcoef.assign((size_t)nv * SW, real(0));
    vwc.assign(plasma ? (size_t)nv * SW * 4 : 0, real(0));
    for (int vl = 0; vl < nv; ++vl) {
      const int sl = own[vl].second;
      vid[vl] = own[vl].first;
      for (int k = 0; k < SW; ++k) {
        const size_t i = (size_t)sl * SW + k, o = (size_t)vl * SW + k;
        vh[o] = locA[ps_edge[i]];
        vcoef[o] = ps_coef[i];
        if (plasma) {
          vj[o] = locB[ps_face[i]];
          for (int c = 0; c < 4; ++c) vwc[o * 4 + c] = ps_wc[i * 4 + c];
        }
      }
    }
    eloc.resize(ne);
    for (int el = 0; el < ne; ++el) {
      const int e = ea + el;
      eloc[el] = make_int4(locA[e], locB[lr[e].x], locB[lr[e].y], 0);
    }
    head[ke_o_vid] = blob_put(T.tab, base, vid.data(), nv * sizeof(int));
    head[ke_o_vh] = blob_put(T.tab, base, vh.data(), vh.size() * sizeof(int));
    head[ke_o_vj] = plasma ? blob_put(T.tab, base, vj.data(), vj.size() * sizeof(int)) : head[ke_o_vh];
    head[ke_o_vcoef] = blob_put(T.tab, base, vcoef.data(), vcoef.size() * (size_t)rb);
    head[ke_o_vwc] = plasma ? blob_put(T.tab, base, vwc.data(), vwc.size() * (size_t)rb) : head[ke_o_vcoef];
    head[ke_o_eloc] = blob_put(T.tab, base, eloc.data(), ne * sizeof(int4));
    head[ke_o_einv] = blob_put(T.tab, base, inv_phi.data() + ea, ne * (size_t)rb);
    head[ke_o_etan] = plasma ? blob_put(T.tab, base, tn.data() + 8 * (size_t)ea, 8 * (size_t)ne * rb) : head[ke_o_einv];
    const int B = (int)(T.tab.size() - base);
    head[ke_nv] = nv;
    head[ke_ea] = ea;
    head[ke_ne] = ne;
    for (const auto& o : own) head[ke_src] |= v_src[o.first] ? 1 : 0;
    for (int e = ea; e < eb; ++e) head[ke_src] |= e_src[e] ? 2 : 0;
    head[ke_o_ht] = B;
    head[ke_o_hr] = head[ke_o_ht] + n_h * Pn * rb;
    head[ke_o_J] = head[ke_o_hr] + n_f * Pm * rb;
    head[ke_o_er] = head[ke_o_J] + (plasma ? n_f * 3 * Pm * rb : 0);
    head[ke_o_et] = head[ke_o_er] + nv * Pn * rb;
    head[ke_o_end] = head[ke_o_et] + ne * Pm * rb;
    const int end = head[ke_o_end];
    if (round128(end) > max_stage) return false;  // the stage would not fit: stop early
    std::memcpy(T.tab.data() + base, head, sizeof(head));
    T.desc.push_back(make_int4(kSrcTab, (int)(base / 16), 0, B));
    add_runs(T.desc, kSrcHt, h_runs, head[ke_o_ht], Pn * rb);
    add_runs(T.desc, kSrcHr, f_runs, head[ke_o_hr], Pm * rb);
    if (plasma) add_runs(T.desc, kSrcJsum, f_runs, head[ke_o_J], 3 * Pm * rb);
    add_runs(T.desc, kSrcEr, v_runs, head[ke_o_er], Pn * rb);
    if (ne > 0) T.desc.push_back(make_int4(kSrcEt, ea, head[ke_o_et], ne * Pm * rb));
    T.dptr.push_back((int)T.desc.size());
    T.stage_bytes = std::max(T.stage_bytes, round128(end));
    if (T.tab.size() / 16 >= (size_t)1 << 31) return false;
  }
  return true;
}

// Fused step through the ring (patch = vertices vlist[vptr[q]..vptr[q+1]) and
// edges eptr[q]..eptr[q+1]; no plasma, no surface impedance).  H edges: the
// owned edges and the slot edges of the owned vertices; H faces: the faces
// beside the owned edges; a face is written by the patch that owns its first
// edge (owner_of_edge).  Stage: blob, er rows (ends of the H edges, which
// include the owned vertices), et rows (H edges and the edges of the H faces),
// ht rows (H edges), hr rows (H faces).
template <typename real>
bool build_pipe_f(PipeTables& T, int n, const std::vector<int>& vptr, const std::vector<int>& vlist,
                  const std::vector<int>& eptr, const std::vector<int>& owner_of_edge, const std::vector<int2>& th,
                  const std::vector<int2>& lr, const std::vector<int4>& fe, int SW, const std::vector<int>& ps_edge,
                  const std::vector<real>& ps_coef, const std::vector<real>& inv_theta, const std::vector<real>& inv_phi,
                  const std::vector<real>& fw, int Pn, int Pm, const std::vector<char>& v_src,
                  const std::vector<char>& e_src, std::vector<int>& locV, std::vector<int>& locE, std::vector<int>& locH,
                  std::vector<int>& locF, int max_stage) {
  using namespace pipe;
  const int rb = (int)sizeof(real);
  std::vector<int> h_ids, f_ids, v_ids, t_ids;
  std::vector<std::pair<int, int>> h_runs, f_runs, v_runs, t_runs;
  std::vector<std::pair<int, int>> own;  // (vertex, slot)
  std::vector<int4> hel, fel, eloc;
  std::vector<int> hid, fid, vid, vh, vel;
  std::vector<real> hinv, fwl, vcoef;
  for (int q = 0; q < n; ++q) {
    const int va = vptr[q], vb = vptr[q + 1], ea = eptr[q], eb = eptr[q + 1], nv = vb - va, ne = eb - ea;
    own.clear();
    for (int sl = va; sl < vb; ++sl) own.push_back({vlist[sl], sl});
    std::sort(own.begin(), own.end());
    h_ids.clear();
    f_ids.clear();
    for (const auto& o : own)
      for (int k = 0; k < SW; ++k) h_ids.push_back(ps_edge[(size_t)o.second * SW + k]);
    for (int e = ea; e < eb; ++e) {
      h_ids.push_back(e);
      f_ids.push_back(lr[e].x);
      f_ids.push_back(lr[e].y);
    }
    sort_unique(h_ids);
    sort_unique(f_ids);
    v_ids.clear();
    t_ids.clear();
    for (const int e : h_ids) {
      v_ids.push_back(th[e].x);
      v_ids.push_back(th[e].y);
      t_ids.push_back(e);
    }
    for (const int f : f_ids) {
      t_ids.push_back(fe[f].x);
      t_ids.push_back(fe[f].y);
      t_ids.push_back(fe[f].z);
    }
    sort_unique(v_ids);
    sort_unique(t_ids);
    int gap = 0, n_v = 0, n_t = 0, n_h = 0, n_f = 0, nd = 0;
    for (;;) {
      n_v = make_runs(v_ids, gap, v_runs, locV);
      n_t = make_runs(t_ids, gap, t_runs, locE);
      n_h = make_runs(h_ids, gap, h_runs, locH);
      n_f = make_runs(f_ids, gap, f_runs, locF);
      nd = 1 + (int)(v_runs.size() + t_runs.size() + h_runs.size() + f_runs.size());
      if (nd <= kMaxDesc || gap >= 64) break;
      gap = 2 * gap + 1;
    }
    if (nd > kMaxDesc) return false;
    const int nhe = (int)h_ids.size(), nhf = (int)f_ids.size();
    hel.resize(nhe);
    hid.resize(nhe);
    hinv.resize(nhe);
    for (int i = 0; i < nhe; ++i) {
      const int e = h_ids[i];
      hel[i] = make_int4(locV[th[e].y], locV[th[e].x], locE[e], locH[e]);
      hid[i] = e | (e >= ea && e < eb ? 0 : kNotOwned);
      hinv[i] = inv_theta[e];
    }
    fel.resize(nhf);
    fid.resize(nhf);
    fwl.resize(4 * (size_t)nhf);
    for (int i = 0; i < nhf; ++i) {
      const int f = f_ids[i];
      fel[i] = make_int4(locE[fe[f].x], locE[fe[f].y], locE[fe[f].z], locF[f]);
      fid[i] = f | (owner_of_edge[fe[f].x] == q ? 0 : kNotOwned);
      for (int c = 0; c < 4; ++c) fwl[4 * (size_t)i + c] = fw[4 * (size_t)f + c];
    }
    vid.assign(nv, 0);
    vel.assign(nv, 0);
    vh.assign((size_t)nv * SW, 0);
    vcoef.assign((size_t)nv * SW, real(0));
    for (int vl = 0; vl < nv; ++vl) {
      const int sl = own[vl].second;
      vid[vl] = own[vl].first;
      vel[vl] = locV[own[vl].first];
      for (int k = 0; k < SW; ++k) {
        const size_t i = (size_t)sl * SW + k, o = (size_t)vl * SW + k;
        vh[o] = locH[ps_edge[i]];
        vcoef[o] = ps_coef[i];
      }
    }
    eloc.resize(ne);
    for (int el = 0; el < ne; ++el) {
      const int e = ea + el;
      eloc[el] = make_int4(locH[e], locF[lr[e].x], locF[lr[e].y], locE[e]);
    }
    const size_t base = T.tab.size();
    int head[kf_head_ints] = {0};
    T.tab.resize(base + sizeof(head), 0);
    head[kf_o_hel] = blob_put(T.tab, base, hel.data(), nhe * sizeof(int4));
    head[kf_o_hinv] = blob_put(T.tab, base, hinv.data(), nhe * (size_t)rb);
    head[kf_o_hid] = blob_put(T.tab, base, hid.data(), nhe * sizeof(int));
    head[kf_o_fel] = blob_put(T.tab, base, fel.data(), nhf * sizeof(int4));
    head[kf_o_fw] = blob_put(T.tab, base, fwl.data(), fwl.size() * (size_t)rb);
    head[kf_o_fid] = blob_put(T.tab, base, fid.data(), nhf * sizeof(int));
    head[kf_o_vid] = blob_put(T.tab, base, vid.data(), nv * sizeof(int));
    head[kf_o_vh] = blob_put(T.tab, base, vh.data(), vh.size() * sizeof(int));
    head[kf_o_vcoef] = blob_put(T.tab, base, vcoef.data(), vcoef.size() * (size_t)rb);
    head[kf_o_vel] = blob_put(T.tab, base, vel.data(), nv * sizeof(int));
    head[kf_o_eloc] = blob_put(T.tab, base, eloc.data(), ne * sizeof(int4));
    head[kf_o_einv] = blob_put(T.tab, base, inv_phi.data() + ea, ne * (size_t)rb);
    const int B = (int)(T.tab.size() - base);
    head[kf_nhe] = nhe;
    head[kf_nhf] = nhf;
    head[kf_nv] = nv;
    head[kf_ea] = ea;
    head[kf_ne] = ne;
    for (const auto& o : own) head[kf_src] |= v_src[o.first] ? 1 : 0;
    for (int e = ea; e < eb; ++e) head[kf_src] |= e_src[e] ? 2 : 0;
    head[kf_o_er] = B;
    head[kf_o_et] = head[kf_o_er] + n_v * Pn * rb;
    head[kf_o_ht] = head[kf_o_et] + n_t * Pm * rb;
    head[kf_o_hr] = head[kf_o_ht] + n_h * Pn * rb;
    head[kf_o_end] = head[kf_o_hr] + n_f * Pm * rb;
    const int end = head[kf_o_end];
    if (round128(end) > max_stage) return false;  // the stage would not fit: stop early
    std::memcpy(T.tab.data() + base, head, sizeof(head));
    T.desc.push_back(make_int4(kSrcTab, (int)(base / 16), 0, B));
    add_runs(T.desc, kSrcEr, v_runs, head[kf_o_er], Pn * rb);
    add_runs(T.desc, kSrcEt, t_runs, head[kf_o_et], Pm * rb);
    add_runs(T.desc, kSrcHt, h_runs, head[kf_o_ht], Pn * rb);
    add_runs(T.desc, kSrcHr, f_runs, head[kf_o_hr], Pm * rb);
    T.dptr.push_back((int)T.desc.size());
    T.stage_bytes = std::max(T.stage_bytes, round128(end));
    if (T.tab.size() / 16 >= (size_t)1 << 31) return false;
  }
  return true;
}

template <typename real>
int build_plan(ifdtd_plan* P, const ifdtd_mesh_desc* M, const ifdtd_grid_desc* G, const ifdtd_physics_desc* X,
               const ifdtd_tuning* tune) {
  Rec<real> R;
  std::memset(&R, 0, sizeof(R));
  const int nV = M->n_vertices, nE = M->n_edges, nF = M->n_faces, L = G->radial_cells;
  if (nV < 4 || nE < 6 || nF < 4 || L < 2) return fail(IFDTD_ERR_ARGUMENT, "mesh or radial grid too small");
  const int Pn = round4(L + 1), Pm = round4(L);
  if ((int64_t)nE * Pn >= (int64_t)1 << 31 || (int64_t)nF * 3 * Pm >= (int64_t)1 << 31)
    return fail(IFDTD_ERR_ARGUMENT, "problem exceeds 2^31 samples per array");
  if (!in_range(M->edges, 2 * (size_t)nE, nV) || !in_range(M->faces, 3 * (size_t)nF, nV) ||
      !in_range(M->face_edges, 3 * (size_t)nF, nE) || !in_range(M->edge_left_faces, nE, nF) ||
      !in_range(M->edge_right_faces, nE, nF))
    return fail(IFDTD_ERR_ARGUMENT, "mesh index table out of range");
  // patch sizes: > 0 as given; 0 (or no tuning) picks, for the pipelined
  // kernels, the largest candidate whose stage fits twice in shared memory,
  // and 32 / 16 faces for the direct kernels
  const bool auto_h = !(tune && tune->faces_per_patch > 0), auto_e = !(tune && tune->e_faces_per_patch > 0);
  int fpp = auto_h ? 32 : tune->faces_per_patch;
  int fpp_e = auto_e ? 16 : tune->e_faces_per_patch;
  const bool fused = tune && tune->fused_step != 0;
  if (tune && (tune->fused_step < 0 || tune->fused_step > 1)) return fail(IFDTD_ERR_ARGUMENT, "fused_step must be 0 or 1");
  if (fused && (X->plasma_species > 0 || X->si_terms > 0))
    return fail(IFDTD_ERR_UNSUPPORTED, "fused_step supports plans without plasma and without surface impedance");
  const int plasma_frame = tune ? tune->plasma_frame : 0;
  if (plasma_frame < 0 || plasma_frame > 2)
    return fail(IFDTD_ERR_ARGUMENT, "plasma_frame must be 0 (auto), 1 (Cartesian) or 2 (face frames)");
  if (plasma_frame == 2 && X->plasma_species > 0 && X->plasma_magnetized)
    return fail(IFDTD_ERR_UNSUPPORTED, "plasma_frame 2 (face frames) supports an unmagnetised plasma only");
  // face frames: the Drude update acts on each component alike, so it is the
  // same in any orthonormal frame; a magnetised update would need B per face
  const bool local = X->plasma_species > 0 && !X->plasma_magnetized && plasma_frame != 1;
  P->plasma_local = local;
  // the fused step replaces both phases; its plan keeps the direct kernels for
  // the single-phase entry points
  const int staging = fused ? 1 : (tune ? tune->staging : 0);
  // fused step: 1 direct gathers; 0 or 2 the ring fed by TMA bulk copies; 3 the ring fed by cp.async
  const int fused_staging = fused && tune ? tune->staging : 0;
  // threads: > 0 as given; 0 picks 320 compute threads for pipelined CTAs and 256 for direct CTAs
  const bool auto_threads = !(tune && tune->threads > 0);
  int threads = auto_threads ? 256 : tune->threads;
  const int producers = (tune && tune->producer_warps > 0) ? tune->producer_warps : 2;
  if (producers > 4) return fail(IFDTD_ERR_ARGUMENT, "producer_warps must be 1 to 4");
  if (!auto_threads && (threads % 32 || threads < 32 || threads + 32 * producers > pipe::kMaxThreads))
    return fail(IFDTD_ERR_ARGUMENT, "threads must be a multiple of 32 and threads + 32 * producer_warps <= 384");
  P->producers = producers;
  if (staging < 0 || staging > 3)
    return fail(IFDTD_ERR_ARGUMENT,
                "staging must be 0 (auto), 1 (direct gathers), 2 (pipeline, TMA bulk copies) or 3 (pipeline, cp.async)");
  P->pipe_copy = staging == 3 ? 1 : 0;
  const int lane_layout = tune ? tune->lane_layout : 0;
  if (lane_layout < 0 || lane_layout > 2)
    return fail(IFDTD_ERR_ARGUMENT, "lane_layout must be 0 (auto), 1 (packed rows) or 2 (rows on 8-lane boundaries)");
  const int e_threads_req = tune ? tune->e_threads : 0;
  // E-phase copy warps: as given; automatic: 4 when both thread counts are
  // automatic (the E stages take about twice the H stages' copies per patch),
  // else the H phase's count
  const int e_producers = (tune && tune->e_producer_warps > 0) ? tune->e_producer_warps
                          : (auto_threads && e_threads_req == 0) ? 4
                                                                  : producers;
  if (e_producers > 4) return fail(IFDTD_ERR_ARGUMENT, "e_producer_warps must be 0 (automatic) or 1 to 4");
  P->e_producers = e_producers;
  if (e_threads_req != 0 &&
      (e_threads_req % 32 || e_threads_req < 32 || e_threads_req + 32 * e_producers > pipe::kWideMaxThreads))
    return fail(IFDTD_ERR_ARGUMENT, "e_threads must be 0 or a multiple of 32 with e_threads + 32 * E producer warps <= 640");
  if (e_threads_req + 32 * e_producers > pipe::kMaxThreads && staging == 3)
    return fail(IFDTD_ERR_ARGUMENT, "wide E-phase CTAs (e_threads + 32 * E producer warps > 384) use TMA bulk copies only");
  const int e_copy_gap = tune ? tune->e_copy_gap : 0;
  if (e_copy_gap < 0 || e_copy_gap > 8) return fail(IFDTD_ERR_ARGUMENT, "e_copy_gap must be 0 to 8");
  const int e_stages_req = tune ? tune->e_stages : 0;
  if (e_stages_req != 0 && (e_stages_req < 2 || e_stages_req > 4))
    return fail(IFDTD_ERR_ARGUMENT, "e_stages must be 0 (auto) or 2 to 4");
  if ((int64_t)std::max(fpp, fpp_e) * 3 * Pn >= (1 << 24)) return fail(IFDTD_ERR_ARGUMENT, "patch too large");
  P->threads = threads;
  // graph_chunk: > 0 steps per captured graph, 0 direct launches, < 0 default
  P->chunk = (tune && tune->graph_chunk >= 0) ? tune->graph_chunk : 32;
  P->nV = nV;
  P->nE = nE;
  P->nF = nF;
  P->L = L;
  P->Pn = Pn;
  P->Pm = Pm;
  DeviceArena& A = P->arena;

  // ---- face frames of the plasma current (float64): e0 along the face
  // centre, e1 along the coordinate axis least aligned with it made
  // orthogonal, e2 = e0 x e1; cnorm = |face centre| ----
  std::vector<double> frame64, cnorm;
  if (local) {
    frame64.assign(9 * (size_t)nF, 0.0);
    cnorm.assign(nF, 0.0);
    for (int f = 0; f < nF; ++f) {
      const double* c = X->face_centers + 3 * (size_t)f;
      const double n = std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
      if (!(n > 0.0) || !std::isfinite(n)) return fail(IFDTD_ERR_ARGUMENT, "face centre of zero or non-finite length");
      const double e0[3] = {c[0] / n, c[1] / n, c[2] / n};
      int a = 0;
      for (int i = 1; i < 3; ++i)
        if (std::fabs(e0[i]) < std::fabs(e0[a])) a = i;
      double e1[3] = {-e0[a] * e0[0], -e0[a] * e0[1], -e0[a] * e0[2]};
      e1[a] += 1.0;
      const double m = std::sqrt(e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2]);
      for (int i = 0; i < 3; ++i) e1[i] /= m;
      const double e2[3] = {e0[1] * e1[2] - e0[2] * e1[1], e0[2] * e1[0] - e0[0] * e1[2], e0[0] * e1[1] - e0[1] * e1[0]};
      double* Q = frame64.data() + 9 * (size_t)f;
      for (int i = 0; i < 3; ++i) {
        Q[i] = e0[i];
        Q[3 + i] = e1[i];
        Q[6 + i] = e2[i];
      }
      cnorm[f] = n;
    }
  }
  // row k of face f's frame applied to a Cartesian vector v
  auto frame_dot = [&](int f, int k, const double* v) {
    const double* Q = frame64.data() + 9 * (size_t)f + 3 * k;
    return Q[0] * v[0] + Q[1] * v[1] + Q[2] * v[2];
  };

  // ---- edges ----
  std::vector<int2> th(nE), lr(nE);
  std::vector<real> inv_theta(nE), inv_phi(nE);
  std::vector<int> owner_e(nE);
  for (int e = 0; e < nE; ++e) {
    th[e] = make_int2((int)M->edges[2 * e], (int)M->edges[2 * e + 1]);
    lr[e] = make_int2((int)M->edge_left_faces[e], (int)M->edge_right_faces[e]);
    inv_theta[e] = (real)(1.0 / M->primal_edge_angles[e]);
    inv_phi[e] = (real)(1.0 / M->dual_edge_angles[e]);
    owner_e[e] = std::min(lr[e].x, lr[e].y);
    if (e > 0 && owner_e[e] < owner_e[e - 1])
      return fail(IFDTD_ERR_ARGUMENT, "edges are not numbered in face-scan order");
  }
  // ---- faces ----
  std::vector<int4> fe(nF), fv(nF);
  std::vector<int> fsign(3 * (size_t)nF);
  std::vector<real> fw(4 * (size_t)nF, real(0));
  for (int f = 0; f < nF; ++f) {
    fe[f] = make_int4((int)M->face_edges[3 * f], (int)M->face_edges[3 * f + 1], (int)M->face_edges[3 * f + 2], 0);
    fv[f] = make_int4((int)M->faces[3 * f], (int)M->faces[3 * f + 1], (int)M->faces[3 * f + 2], 0);
    const double inv_a = 1.0 / M->face_solid_angles[f];
    for (int i = 0; i < 3; ++i) {
      const int64_t s = M->face_edge_signs[3 * f + i];
      if (s != 1 && s != -1) return fail(IFDTD_ERR_ARGUMENT, "face edge signs must be +1 or -1");
      fsign[3 * f + i] = (int)s;
      fw[4 * f + i] = (real)((double)s * M->primal_edge_angles[M->face_edges[3 * f + i]] * inv_a);
    }
  }
  // ---- vertex incidence in reference slot order: tail uses, then head uses ----
  std::vector<int> deg(nV, 0);
  for (int e = 0; e < nE; ++e) {
    deg[th[e].x]++;
    deg[th[e].y]++;
  }
  std::vector<int> v_off(nV + 1, 0);
  for (int v = 0; v < nV; ++v) v_off[v + 1] = v_off[v] + deg[v];
  std::vector<int> fill(v_off.begin(), v_off.end() - 1);
  std::vector<int> v_edge(2 * (size_t)nE), v_sign(2 * (size_t)nE);
  std::vector<double> v_coef(2 * (size_t)nE);
  for (int pass = 0; pass < 2; ++pass)
    for (int e = 0; e < nE; ++e) {
      const int v = pass == 0 ? th[e].x : th[e].y;
      const int q = fill[v]++;
      v_edge[q] = e;
      v_sign[q] = pass == 0 ? 1 : -1;
      v_coef[q] = (pass == 0 ? 1.0 : -1.0) * M->dual_edge_angles[e] / M->dual_cell_solid_angles[v];
    }
  // ---- patches: faces [p*fpp, (p+1)*fpp), edges by lowest adjacent face, vertices by lowest incident face ----
  std::vector<int> owner_v(nV, nF);
  for (int f = 0; f < nF; ++f) {
    owner_v[fv[f].x] = std::min(owner_v[fv[f].x], f);
    owner_v[fv[f].y] = std::min(owner_v[fv[f].y], f);
    owner_v[fv[f].z] = std::min(owner_v[fv[f].z], f);
  }
  for (int v = 0; v < nV; ++v)
    if (owner_v[v] >= nF) return fail(IFDTD_ERR_ARGUMENT, "vertex without incident face");
  struct Own {
    int fpp = 0, n = 0;
    std::vector<int> eptr, vptr, vlist;
  };
  auto ownership = [&](int f_per) {
    Own o;
    o.fpp = f_per;
    o.n = (nF + f_per - 1) / f_per;
    o.eptr.assign(o.n + 1, 0);
    int e = 0;
    for (int q = 0; q <= o.n; ++q) {
      const int bound = std::min(q * f_per, nF);
      while (e < nE && owner_e[e] < bound) ++e;
      o.eptr[q] = (q == o.n) ? nE : e;
    }
    o.vptr.assign(o.n + 1, 0);
    o.vlist.assign(nV, 0);
    for (int v = 0; v < nV; ++v) o.vptr[owner_v[v] / f_per + 1]++;
    for (int q = 0; q < o.n; ++q) o.vptr[q + 1] += o.vptr[q];
    std::vector<int> cursor(o.vptr.begin(), o.vptr.end() - 1);
    for (int v = 0; v < nV; ++v) o.vlist[cursor[owner_v[v] / f_per]++] = v;
    return o;
  };
  // ownership with arbitrary patch boundaries: patch q owns faces [bounds[q], bounds[q+1])
  // and the edges and vertices whose lowest adjacent / incident face lies there
  auto ownership_bounds = [&](const std::vector<int>& bounds) {
    Own o;
    o.fpp = 0;
    o.n = (int)bounds.size() - 1;
    o.eptr.assign(o.n + 1, nE);
    int e = 0;
    for (int q = 0; q < o.n; ++q) {
      while (e < nE && owner_e[e] < bounds[q]) ++e;
      o.eptr[q] = e;
    }
    std::vector<int> patch_of_face(nF);
    for (int q = 0; q < o.n; ++q)
      for (int f = bounds[q]; f < bounds[q + 1]; ++f) patch_of_face[f] = q;
    o.vptr.assign(o.n + 1, 0);
    o.vlist.assign(nV, 0);
    for (int v = 0; v < nV; ++v) o.vptr[patch_of_face[owner_v[v]] + 1]++;
    for (int q = 0; q < o.n; ++q) o.vptr[q + 1] += o.vptr[q];
    std::vector<int> cursor(o.vptr.begin(), o.vptr.end() - 1);
    for (int v = 0; v < nV; ++v) o.vlist[cursor[patch_of_face[owner_v[v]]]++] = v;
    return o;
  };
  Own oh = ownership(fpp), oe = ownership(fpp_e);
  // ---- fixed-width vertex slots in vlist order (reference slot order, zero-padded) ----
  int maxdeg = 0;
  for (int v = 0; v < nV; ++v) maxdeg = std::max(maxdeg, deg[v]);
  const int MD = maxdeg <= 6 ? 6 : (maxdeg <= 12 ? 12 : 0);
  if (MD == 0) return fail(IFDTD_ERR_UNSUPPORTED, "vertex degree above 12 is not supported");
  const int SW = round4(MD);
  P->maxdeg = MD;
  struct Slots {
    std::vector<int> edge, face;
    std::vector<real> coef, wc;
  };
  // slot tables of the vertices in the order `vlist` lists them; false on a bad vertex face table
  auto build_slots = [&](const std::vector<int>& vlist, Slots& out) {
    out.edge.assign((size_t)nV * SW, 0);
    out.coef.assign((size_t)nV * SW, real(0));
    for (int sl = 0; sl < nV; ++sl) {
      const int v = vlist[sl];
      const int q0 = v_off[v], n = v_off[v + 1] - q0;
      for (int q = 0; q < SW; ++q) {
        out.edge[(size_t)sl * SW + q] = v_edge[q0 + (q < n ? q : 0)];
        out.coef[(size_t)sl * SW + q] = q < n ? (real)v_coef[q0 + q] : real(0);
      }
    }
    out.face.clear();
    out.wc.clear();
    if (X->plasma_species > 0) {
      const int W = X->vertex_face_width;
      out.face.assign((size_t)nV * SW, 0);
      out.wc.assign((size_t)nV * SW * 4, real(0));
      for (int sl = 0; sl < nV; ++sl) {
        const int v = vlist[sl];
        int n = 0, first = -1;
        for (int q = 0; q < W; ++q) {
          const double w = X->vertex_face_weights[(size_t)v * W + q];
          if (w == 0.0) continue;
          const int64_t f = X->vertex_faces[(size_t)v * W + q];
          if (f < 0 || f >= nF || n >= MD) return false;
          if (first < 0) first = (int)f;
          out.face[(size_t)sl * SW + n] = (int)f;
          if (local)  // face frames: the slots' weights packed first, w * |centre| (its e0 component)
            out.wc[(size_t)sl * SW * 4 + n] = (real)(w * cnorm[f]);
          else
            for (int c = 0; c < 3; ++c) out.wc[((size_t)sl * SW + n) * 4 + c] = (real)(w * X->face_centers[3 * f + c]);
          ++n;
        }
        for (int q = n; q < SW; ++q) out.face[(size_t)sl * SW + q] = first < 0 ? 0 : first;
      }
    }
    return true;
  };
  // E-phase patch boundaries whose staged bytes (the pipelined E stage layout,
  // before 16-byte run bridging) stay within `cap`: faces are scanned in order
  // and a patch closes before the face whose owned vertices and edges would
  // overflow it.
  std::vector<int> vtx_by_owner_off(nF + 1, 0), vtx_by_owner;
  for (int v = 0; v < nV; ++v) vtx_by_owner_off[owner_v[v] + 1]++;
  for (int f = 0; f < nF; ++f) vtx_by_owner_off[f + 1] += vtx_by_owner_off[f];
  vtx_by_owner.assign(nV, 0);
  {
    std::vector<int> cur(vtx_by_owner_off.begin(), vtx_by_owner_off.end() - 1);
    for (int v = 0; v < nV; ++v) vtx_by_owner[cur[owner_v[v]]++] = v;
  }
  auto balanced_e_bounds = [&](int cap, bool with_plasma, int rb) {
    std::vector<int> bounds{0};
    std::vector<int> stamp_e(nE, -1), stamp_f(nF, -1);
    int patch = 0, n_ht = 0, n_f = 0, nv = 0, ne = 0;
    const int W = X->vertex_face_width;
    auto a16 = [](long b) { return (b + 15) / 16 * 16; };
    auto bytes = [&](int h, int fcount, int v, int e) {
      long blob = 16L * ((pipe::ke_head_ints * 4 + 15) / 16) + a16(4L * v) + a16(4L * v * SW) * (with_plasma ? 2 : 1) + a16((long)rb * v * SW) +
                  (with_plasma ? a16(4L * rb * v * SW) : 0) + a16(16L * e) + a16((long)rb * e) +
                  (with_plasma ? a16(8L * rb * e) : 0);
      long rows = (long)rb * ((long)h * Pn + (long)fcount * Pm * (with_plasma ? 4 : 1) + (long)v * Pn + (long)e * Pm);
      return (blob + rows + 127) / 128 * 128;
    };
    int e_cursor = 0;
    std::vector<int> touched_e, touched_f;
    for (int f = 0; f < nF; ++f) {
      const int e0 = e_cursor;
      while (e_cursor < nE && owner_e[e_cursor] == f) ++e_cursor;
      for (int pass = 0; pass < 2; ++pass) {
        // pass 0: count what face f's entities add; pass 1: commit them
        int dh = 0, df = 0;
        const int mark = pass == 0 ? -2 - patch : patch;  // pass-0 marks are undone below
        touched_e.clear();
        touched_f.clear();
        auto add_e = [&](int id) {
          if (stamp_e[id] != patch && stamp_e[id] != -2 - patch) {
            stamp_e[id] = mark;
            ++dh;
            if (pass == 0) touched_e.push_back(id);
          } else if (pass == 1 && stamp_e[id] != patch) {
            stamp_e[id] = patch;
          }
        };
        auto add_f = [&](int id) {
          if (stamp_f[id] != patch && stamp_f[id] != -2 - patch) {
            stamp_f[id] = mark;
            ++df;
            if (pass == 0) touched_f.push_back(id);
          } else if (pass == 1 && stamp_f[id] != patch) {
            stamp_f[id] = patch;
          }
        };
        for (int k = vtx_by_owner_off[f]; k < vtx_by_owner_off[f + 1]; ++k) {
          const int v = vtx_by_owner[k];
          for (int q = v_off[v]; q < v_off[v + 1]; ++q) add_e(v_edge[q]);
          if (with_plasma)
            for (int q = 0; q < W; ++q)
              if (X->vertex_face_weights[(size_t)v * W + q] != 0.0) add_f((int)X->vertex_faces[(size_t)v * W + q]);
        }
        for (int e = e0; e < e_cursor; ++e) {
          add_e(e);
          add_f(lr[e].x);
          add_f(lr[e].y);
        }
        const int dv = vtx_by_owner_off[f + 1] - vtx_by_owner_off[f], de = e_cursor - e0;
        if (pass == 0) {
          for (int id : touched_e) stamp_e[id] = -1;
          for (int id : touched_f) stamp_f[id] = -1;
          if ((nv + ne) > 0 && bytes(n_ht + dh, n_f + df, nv + dv, ne + de) > cap) {
            bounds.push_back(f);  // close the patch before face f
            ++patch;
            n_ht = n_f = nv = ne = 0;
          }
        } else {
          n_ht += dh;
          n_f += df;
          nv += dv;
          ne += de;
        }
      }
    }
    bounds.push_back(nF);
    return bounds;
  };
  Slots slots;
  if (!build_slots(oe.vlist, slots))
    return fail(IFDTD_ERR_ARGUMENT, "vertex face table out of range or wider than the vertex degree");

  const int S = std::max(0, X->plasma_species);
  const bool plasma = S > 0;

  // ---- fused step: E patches with their halo edge and face lists ----
  PipeTables tf_tab;  // the ring's descriptors and blobs (uploaded with the E-phase tables)
  if (fused) {
    if (P->chunk % 2) return fail(IFDTD_ERR_ARGUMENT, "fused_step needs an even graph_chunk");
    std::vector<int> patch_of_edge(nE), stamp_e(nE), stamp_f(nF), loc_e(nE), loc_f(nF);
    std::vector<int> halo_e, own_f, halo_f;
    // the halo tables of ownership o (slots sl in o.vlist order); false if a
    // table would be inconsistent
    auto build_fused = [&](const Own& o, const Slots& sl, std::vector<int4>& fpatch, std::vector<int>& hedge,
                           std::vector<int>& hface, std::vector<int>& vslot, std::vector<int2>& eface,
                           size_t& max_rows) {
      for (int q = 0; q < o.n; ++q)
        for (int e = o.eptr[q]; e < o.eptr[q + 1]; ++e) patch_of_edge[e] = q;
      std::fill(stamp_e.begin(), stamp_e.end(), -1);
      std::fill(stamp_f.begin(), stamp_f.end(), -1);
      fpatch.assign(o.n + 1, make_int4(0, 0, 0, 0));
      hedge.clear();
      hface.clear();
      vslot.assign((size_t)nV * SW, 0);
      eface.assign(nE, make_int2(0, 0));
      max_rows = 0;
      size_t owned_faces = 0;
      for (int q = 0; q < o.n; ++q) {
        const int e0 = o.eptr[q], e1 = o.eptr[q + 1];
        const int he0 = (int)hedge.size(), hf0 = (int)hface.size();
        // owned edges first, in order, then the other edges of the owned vertices
        for (int e = e0; e < e1; ++e) {
          stamp_e[e] = q;
          loc_e[e] = (int)hedge.size() - he0;
          hedge.push_back(e);
        }
        halo_e.clear();
        for (int k = o.vptr[q]; k < o.vptr[q + 1]; ++k) {
          const int v = o.vlist[k];
          for (int i = v_off[v]; i < v_off[v + 1]; ++i) {
            const int e = v_edge[i];
            if (stamp_e[e] != q) {
              stamp_e[e] = q;
              halo_e.push_back(e);
            }
          }
        }
        std::sort(halo_e.begin(), halo_e.end());
        for (const int e : halo_e) {
          loc_e[e] = (int)hedge.size() - he0;
          hedge.push_back(e);
        }
        // faces beside the owned edges: first those whose first edge the patch owns (it writes them)
        own_f.clear();
        halo_f.clear();
        for (int e = e0; e < e1; ++e)
          for (const int f : {lr[e].x, lr[e].y})
            if (stamp_f[f] != q) {
              stamp_f[f] = q;
              (patch_of_edge[fe[f].x] == q ? own_f : halo_f).push_back(f);
            }
        std::sort(own_f.begin(), own_f.end());
        std::sort(halo_f.begin(), halo_f.end());
        for (const auto* list : {&own_f, &halo_f})
          for (const int f : *list) {
            loc_f[f] = (int)hface.size() - hf0;
            hface.push_back(f);
          }
        owned_faces += own_f.size();
        fpatch[q] = make_int4(he0, e1 - e0, hf0, (int)own_f.size());
        for (int k = o.vptr[q]; k < o.vptr[q + 1]; ++k)
          for (int j = 0; j < SW; ++j) {
            const int e = sl.edge[(size_t)k * SW + j];
            if (stamp_e[e] != q) return false;
            vslot[(size_t)k * SW + j] = loc_e[e];
          }
        for (int e = e0; e < e1; ++e) eface[e] = make_int2(loc_f[lr[e].x], loc_f[lr[e].y]);
        const size_t rows = ((size_t)(hedge.size() - he0) * Pn + (size_t)(hface.size() - hf0) * Pm) * sizeof(real);
        max_rows = std::max(max_rows, rows);
      }
      fpatch[o.n] = make_int4((int)hedge.size(), 0, (int)hface.size(), 0);
      return owned_faces == (size_t)nF;  // every face written by exactly one patch
    };
    const int lreals = layer_reals(Pn, Pm, X->coef_rows_er != 1, 0, 0, 0, 0);
    const size_t layer_bytes = (size_t)(lreals + 3) / 4 * 4 * sizeof(real);
    bool done = false;
    if (fused_staging != 1) {
      // the ring: the largest patch whose stage fits twice beside the per-layer rows
      const int f_budget = kSmemPerBlock - (int)sizeof(Rec<real>) - 1024 - pipe::layer_block_bytes(lreals, (int)sizeof(real));
      const int W = P->e_producers;
      const int f_threads = e_threads_req > 0 ? e_threads_req : pipe::kMaxThreads - 32 * W;
      const int row_quads = std::max(Pn, Pm) / (16 / (int)sizeof(real));
      if (f_threads + 32 * W > pipe::kMaxThreads)
        return fail(IFDTD_ERR_ARGUMENT, "fused step: e_threads + 32 * E producer warps must not exceed 384");
      std::vector<char> v_src(nV, 0), e_src(nE, 0);
      for (int q = 0; q < X->n_src_er; ++q) v_src[X->src_er_vertex[q]] = 1;
      for (int q = 0; q < X->n_src_et; ++q) e_src[X->src_et_edge[q]] = 1;
      std::vector<int> locV(nV), locE(nE), locH(nE), locF(nF);
      std::vector<int> cand_f = auto_e ? std::vector<int>{64, 48, 32, 24, 16, 8} : std::vector<int>{fpp_e};
      if (row_quads > f_threads) cand_f.clear();
      for (const int c : cand_f) {
        Own o = ownership(c);
        Slots sl;
        if (!build_slots(o.vlist, sl)) break;
        for (int q = 0; q < o.n; ++q)
          for (int e = o.eptr[q]; e < o.eptr[q + 1]; ++e) patch_of_edge[e] = q;
        PipeTables t;
        const bool ok = build_pipe_f<real>(t, o.n, o.vptr, o.vlist, o.eptr, patch_of_edge, th, lr, fe, SW, sl.edge,
                                           sl.coef, inv_theta, inv_phi, fw, Pn, Pm, v_src, e_src, locV, locE, locH,
                                           locF, f_budget / 2);
        if (!ok || 2 * t.stage_bytes > f_budget || !descriptors_valid(t, (int)sizeof(real), Pn, Pm, 0, nV, nE, nF, 0))
          continue;
        fpp_e = c;
        oe = std::move(o);
        slots = std::move(sl);
        P->kf_stage = t.stage_bytes;
        P->kf_stages = std::min(pipe::kMaxStages, f_budget / t.stage_bytes);
        P->kf_smem = (size_t)pipe::layer_block_bytes(lreals, (int)sizeof(real)) + (size_t)P->kf_stages * P->kf_stage;
        P->kf_threads = f_threads;
        P->kf_producers = W;
        const int wide = std::max((Pn / (int)(16 / sizeof(real)) + 7) & ~7, (Pm / (int)(16 / sizeof(real)) + 7) & ~7);
        P->kf_lanes = lane_layout == 2 && wide <= f_threads ? 1 : 0;
        P->pipe_copy = fused_staging == 3 ? 1 : 0;
        P->kf_cost.assign(o.n, 0.f);
        for (int q = 0; q < o.n; ++q)
          for (int d = t.dptr[q]; d < t.dptr[q + 1]; ++d) P->kf_cost[q] += (float)t.desc[d].w;
        tf_tab = std::move(t);
        P->fused_pipe = true;
        done = true;
        break;
      }
      if (!done && fused_staging >= 2)
        return fail(IFDTD_ERR_UNSUPPORTED, "fused step: no patch's stage fits twice in shared memory");
    }
    const size_t budget = 110 * 1024;  // direct gathers: two CTAs per SM
    std::vector<int> cand = done ? std::vector<int>{} : auto_e ? std::vector<int>{128, 64, 32, 16} : std::vector<int>{fpp_e};
    std::vector<int4> fpatch;
    std::vector<int> hedge, hface, vslot;
    std::vector<int2> eface;
    for (const int c : cand) {
      Own o = ownership(c);
      Slots sl;
      size_t max_rows = 0;
      if (!build_slots(o.vlist, sl) || !build_fused(o, sl, fpatch, hedge, hface, vslot, eface, max_rows))
        return fail(IFDTD_ERR_ARGUMENT, "fused step tables are inconsistent with the mesh");
      if (layer_bytes + max_rows > (auto_e ? budget : (size_t)kSmemPerBlock - sizeof(Rec<real>) - 1024)) continue;
      fpp_e = c;
      oe = std::move(o);
      slots = std::move(sl);
      P->fused_smem = layer_bytes + max_rows;
      done = true;
      break;
    }
    if (!done) return fail(IFDTD_ERR_UNSUPPORTED, "fused step: no patch's halo rows fit in shared memory");
    cudaError_t e = cudaSuccess;
    if (!P->fused_pipe) {
      FusedTables& F = P->fused_tab;
      e = A.upload(fpatch, &F.patch);
      if (e == cudaSuccess) e = A.upload(hedge, &F.hedge);
      if (e == cudaSuccess) e = A.upload(hface, &F.hface);
      if (e == cudaSuccess) e = A.upload(vslot, &F.vslot);
      if (e == cudaSuccess) e = A.upload(eface, &F.eface);
    }
    const size_t rows[4] = {(size_t)nV * Pn, (size_t)nE * Pm, (size_t)nF * Pm, (size_t)nE * Pn};
    for (int i = 0; i < 4 && e == cudaSuccess; ++i) {
      P->fb_bytes[i] = rows[i] * sizeof(real);
      e = A.alloc(P->fb_bytes[i], &P->fb[i]);
      if (e == cudaSuccess) e = cudaMemset(P->fb[i], 0, P->fb_bytes[i]);
    }
    if (e != cudaSuccess) return fail(IFDTD_ERR_CUDA, std::string("fused step tables: ") + cudaGetErrorString(e));
    P->fused = true;
  }

  // ---- radial metric rows, zero padded to Pn / Pm ----
  const double* r = G->radii_m;
  std::vector<real> invr(Pn, 0), rr(Pn, 0), invcd(Pn, 0), mid(Pm, 0), invm(Pm, 0), invdr(Pm, 0);
  std::vector<double> m(L);
  for (int k = 0; k <= L; ++k) {
    if (!(r[k] > 0.0) || (k > 0 && !(r[k] > r[k - 1]))) return fail(IFDTD_ERR_ARGUMENT, "radii must increase");
    invr[k] = (real)(1.0 / r[k]);
    rr[k] = (real)r[k];
  }
  for (int j = 0; j < L; ++j) {
    m[j] = 0.5 * (r[j] + r[j + 1]);
    mid[j] = (real)m[j];
    invm[j] = (real)(1.0 / m[j]);
    invdr[j] = (real)(1.0 / (r[j + 1] - r[j]));
  }
  invcd[0] = (real)(2.0 / (r[1] - r[0]));
  invcd[L] = (real)(2.0 / (r[L] - r[L - 1]));
  for (int k = 1; k < L; ++k) invcd[k] = (real)(1.0 / (m[k] - m[k - 1]));
  // fused rows (float64 products, zero beyond the last node / midpoint):
  //   hA = dt/(mu0 r); hU, hD: weights of Et[k] and Et[k-1] in dt/mu0 (1/r) d(m Et)/dr
  //   (thin shell: d Et / dr) with zero (PEC-odd) ghosts; hC = dt/(mu0 m);
  //   vwl, vwu: node weights of the midpoints below / above (one-sided at the
  //   boundary nodes); eU, eD: weights of Ht[j+1] and Ht[j] in (1/m) d(r Ht)/dr
  //   (thin shell: d Ht / dr).
  std::vector<real> hA(Pn, 0), hU(Pn, 0), hD(Pn, 0), vwl(Pn, 0), vwu(Pn, 0), hC(Pm, 0), eU(Pm, 0), eD(Pm, 0);
  {
    const double dtmu = G->time_step_s / 1.256637062120e-6;
    const bool full = G->full_spherical != 0;
    std::vector<double> cd(L + 1);
    cd[0] = 2.0 / (r[1] - r[0]);
    cd[L] = 2.0 / (r[L] - r[L - 1]);
    for (int k = 1; k < L; ++k) cd[k] = 1.0 / (m[k] - m[k - 1]);
    for (int k = 0; k <= L; ++k) {
      hA[k] = (real)(dtmu / r[k]);
      const double w = full ? dtmu * cd[k] / r[k] : dtmu * cd[k];
      if (k < L) hU[k] = (real)(full ? w * m[k] : w);
      if (k >= 1) hD[k] = (real)(full ? w * m[k - 1] : w);
      vwl[k] = (real)(k == 0 ? 0.0 : (k == L ? 1.0 : 0.5));
      vwu[k] = (real)(k == 0 ? 1.0 : (k == L ? 0.0 : 0.5));
    }
    for (int j = 0; j < L; ++j) {
      const double idr = 1.0 / (r[j + 1] - r[j]);
      hC[j] = (real)(dtmu / m[j]);
      eU[j] = (real)(full ? r[j + 1] * idr / m[j] : idr);
      eD[j] = (real)(full ? r[j] * idr / m[j] : idr);
    }
  }

  // ---- loss coefficients, rows padded to Pn / Pm ----
  if (!(X->coef_rows_er == 1 || X->coef_rows_er == nV) || !(X->coef_rows_et == 1 || X->coef_rows_et == nE))
    return fail(IFDTD_ERR_ARGUMENT, "coefficient rows must be 1 or the entity count");
  if ((X->coef_rows_er == 1) != (X->coef_rows_et == 1))
    return fail(IFDTD_ERR_ARGUMENT, "er and et coefficients must both be compressed or both full");
  auto pad_rows = [](const double* src, int rows, int cols, int pitch) {
    std::vector<real> out((size_t)rows * pitch, real(0));
    for (int i = 0; i < rows; ++i)
      for (int j = 0; j < cols; ++j) out[(size_t)i * pitch + j] = (real)src[(size_t)i * cols + j];
    return out;
  };

  // ---- sources ----
  if (X->n_src_er < 0 || X->n_src_er > IFDTD_MAX_SOURCES || X->n_src_et < 0 || X->n_src_et > IFDTD_MAX_SOURCES)
    return fail(IFDTD_ERR_ARGUMENT, "too many source supports");
  static_assert(kMaxSources >= IFDTD_MAX_SOURCES, "record source table too small");
  for (int s = 0; s < X->n_src_er; ++s) {
    if (X->src_er_vertex[s] < 0 || X->src_er_vertex[s] >= nV || X->src_er_layer[s] < 0 || X->src_er_layer[s] > L)
      return fail(IFDTD_ERR_ARGUMENT, "vertical source support out of range");
    R.src_er_v[s] = (int)X->src_er_vertex[s];
    R.src_er_k[s] = (int)X->src_er_layer[s];
    R.src_er_c[s] = (real)X->src_er_coef[s];
  }
  for (int s = 0; s < X->n_src_et; ++s) {
    if (X->src_et_edge[s] < 0 || X->src_et_edge[s] >= nE || X->src_et_layer[s] < 0 || X->src_et_layer[s] >= L)
      return fail(IFDTD_ERR_ARGUMENT, "tangential source support out of range");
    R.src_et_e[s] = (int)X->src_et_edge[s];
    R.src_et_j[s] = (int)X->src_et_layer[s];
    R.src_et_c[s] = (real)X->src_et_coef[s];
  }

  // ---- upload ----
#define UP(vec, field)                                                                                  \
  do {                                                                                                  \
    cudaError_t _e = A.upload(vec, &R.field);                                                           \
    if (_e != cudaSuccess)                                                                              \
      return fail(IFDTD_ERR_CUDA, std::string("upload ") + #field + ": " + cudaGetErrorString(_e));     \
  } while (0)
  UP(th, edge_th);
  UP(lr, edge_lr);
  UP(inv_theta, inv_theta);
  UP(inv_phi, inv_phi);
  UP(fe, face_e);
  UP(fv, face_v);
  UP(fw, face_w);
  UP(invr, invr);
  UP(rr, rr);
  UP(mid, mid);
  UP(invm, invm);
  UP(invdr, invdr);
  UP(invcd, invcd);
  UP(hA, hA);
  UP(hU, hU);
  UP(hD, hD);
  UP(hC, hC);
  UP(vwl, vwl);
  UP(vwu, vwu);
  UP(eU, eU);
  UP(eD, eD);
  {
    auto ca = pad_rows(X->ca_er, X->coef_rows_er, L + 1, Pn), cb = pad_rows(X->cb_er, X->coef_rows_er, L + 1, Pn);
    auto ct = pad_rows(X->ca_et, X->coef_rows_et, L, Pm), cu = pad_rows(X->cb_et, X->coef_rows_et, L, Pm);
    UP(ca, ca_er);
    UP(cb, cb_er);
    UP(ct, ca_et);
    UP(cu, cb_et);
  }
  {
    cudaError_t e1 = A.upload(fsign, &P->face_sign);
    cudaError_t e2 = A.upload(v_sign, &P->v_sign);
    cudaError_t e3 = A.upload(v_off, &P->v_off);
    cudaError_t e4 = A.upload(v_edge, &P->v_edge);
    if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess || e4 != cudaSuccess)
      return fail(IFDTD_ERR_CUDA, "upload of primitive tables failed");
  }
  P->edge_th = R.edge_th;
  P->edge_lr = R.edge_lr;
  P->face_e = R.face_e;

  // ---- surface impedance ----
  P->T = X->si_terms;
  if (X->si_terms < 0 || X->si_terms > 256) return fail(IFDTD_ERR_ARGUMENT, "surface impedance terms out of range");
  if (X->si_terms > 0) {
    const int T = X->si_terms;
    auto sc = cast<real>(X->si_scale, nE), dc = cast<real>(X->si_decay, T), dr = cast<real>(X->si_drive, T),
         hw = cast<real>(X->si_history, T);
    double hsum = 0.0;
    for (int p = 0; p < T; ++p) hsum += X->si_history[p];
    UP(sc, si_scale);
    UP(dc, si_decay);
    UP(dr, si_drive);
    UP(hw, si_hist);
    R.si_metric = (real)X->si_metric;
    R.si_kappa = (real)(2.0 * G->time_step_s / (1.256637062120e-6 * (r[1] - r[0])));
    R.si_hist_sum = (real)hsum;
  }

  // ---- plasma ----
  std::vector<real> pl, tn;  // (F, 12) reconstruction rows, (E, 8) edge tangents
  P->S = X->plasma_species;
  if (X->plasma_species < 0 || X->plasma_species > IFDTD_MAX_SPECIES)
    return fail(IFDTD_ERR_ARGUMENT, "plasma species count out of range");
  if (X->plasma_species > 0) {
    const int S = X->plasma_species, rows = X->plasma_rows;
    if (!(rows == 1 || rows == nF)) return fail(IFDTD_ERR_ARGUMENT, "plasma rows must be 1 or F");
    P->plasma = true;
    pl.assign(12 * (size_t)nF, real(0));
    tn.assign(8 * (size_t)nE, real(0));
    if (local) {
      // reconstruction rows and centre in the face's frame (the centre is
      // |centre| e0); edge tangents in their faces' frames, components 1 and 2
      // (the tangents lie in the faces' tangent planes)
      std::vector<real> fr(12 * (size_t)nF, real(0));
      for (int f = 0; f < nF; ++f) {
        for (int i = 0; i < 3; ++i) {
          const double* row = X->plasma_reconstruction + 9 * (size_t)f + 3 * i;
          for (int k = 0; k < 3; ++k) pl[12 * (size_t)f + 4 * i + k] = (real)frame_dot(f, k, row);
          pl[12 * (size_t)f + 4 * i + 3] = (real)(i == 0 ? cnorm[f] : 0.0);
          for (int c = 0; c < 3; ++c) fr[12 * (size_t)f + 4 * i + c] = (real)frame64[9 * (size_t)f + 3 * i + c];
        }
      }
      for (int e = 0; e < nE; ++e) {
        const int fl = (int)M->edge_left_faces[e], fq = (int)M->edge_right_faces[e];
        const double* tl = X->plasma_tangent_left + 3 * (size_t)e;
        const double* tq = X->plasma_tangent_right + 3 * (size_t)e;
        tn[8 * (size_t)e + 0] = (real)frame_dot(fl, 1, tl);
        tn[8 * (size_t)e + 1] = (real)frame_dot(fl, 2, tl);
        tn[8 * (size_t)e + 2] = (real)frame_dot(fq, 1, tq);
        tn[8 * (size_t)e + 3] = (real)frame_dot(fq, 2, tq);
      }
      UP(fr, frame);
      P->d_frame = R.frame;
    } else {
      for (int f = 0; f < nF; ++f)
        for (int i = 0; i < 3; ++i) {
          for (int c = 0; c < 3; ++c) pl[12 * (size_t)f + 4 * i + c] = (real)X->plasma_reconstruction[9 * (size_t)f + 3 * i + c];
          pl[12 * (size_t)f + 4 * i + 3] = (real)X->face_centers[3 * (size_t)f + i];
        }
      for (int e = 0; e < nE; ++e)
        for (int c = 0; c < 3; ++c) {
          tn[8 * (size_t)e + c] = (real)X->plasma_tangent_left[3 * (size_t)e + c];
          tn[8 * (size_t)e + 4 + c] = (real)X->plasma_tangent_right[3 * (size_t)e + c];
        }
    }
    auto pc = pad_rows(X->plasma_coef, S * 6 * rows, L, Pm);
    UP(pl, face_pl);
    UP(tn, tan);
    UP(pc, pcoef);
    if (X->plasma_magnetized) {
      std::vector<real> bd((size_t)rows * 3 * Pm, real(0));  // component-major (rows, 3, Pm)
      for (int i = 0; i < rows; ++i)
        for (int j = 0; j < L; ++j)
          for (int c = 0; c < 3; ++c) bd[((size_t)i * 3 + c) * Pm + j] = (real)X->plasma_bdir[((size_t)i * L + j) * 3 + c];
      UP(bd, bdir);
    }
    if (S > 1) {
      cudaError_t e = A.alloc((size_t)nF * 3 * Pm * sizeof(real), &P->d_jtot);
      if (e != cudaSuccess) return fail(IFDTD_ERR_CUDA, "allocation of summed plasma current failed");
      R.Jtot = (real*)P->d_jtot;
    }
  }

  // ---- pipelined kernels: copy descriptors and table blobs per patch ----
  const int layer_block = pipe::layer_block_bytes(
      layer_reals(Pn, Pm, X->coef_rows_er != 1, S, X->plasma_rows == nF && nF != 1, X->plasma_magnetized != 0,
                  X->si_terms),
      (int)sizeof(real));
  // static shared memory of the pipelined kernels: the record, 2 x 8 barriers
  // and the abort flag, well inside 1 KiB besides the record
  const int stage_budget = kSmemPerBlock - (int)sizeof(Rec<real>) - 1024 - layer_block;
  if (staging != 1) {
    PipeTables th_tab, te_tab;
    std::vector<int> locA(std::max(nV, std::max(nE, nF)), 0), locB(std::max(nE, nF), 0);
    // the pipelined consumers give every compute thread a fixed radial quad,
    // so no row may have more quads than the CTA has compute threads (at least
    // 256 when the count is automatic)
    const int row_quads = std::max(Pn, Pm) / (16 / (int)sizeof(real));
    const bool quads_fit = row_quads <= (auto_threads ? 256 : threads) && (e_threads_req == 0 || row_quads <= e_threads_req);
    std::vector<int> h_cand = auto_h ? std::vector<int>{256, 128, 64, 32, 16, 8} : std::vector<int>{fpp};
    if (!quads_fit) h_cand.clear();
    for (const int c : h_cand) {
      Own o = ownership(c);
      PipeTables t;
      const bool ok =
          build_pipe_h<real>(t, o.n, c, nF, o.eptr, th, fe, fv, inv_theta, fw, pl, S, Pn, Pm, X->si_terms,
                             X->si_scale, locA, locB, stage_budget / 2);
      if (ok && 2 * t.stage_bytes <= stage_budget) {
        P->pipe_h_ok = true;
        fpp = c;
        oh = std::move(o);
        th_tab = std::move(t);
        break;
      }
    }
    // E phase: balanced patches for two, then three stages; then fixed face counts
    std::vector<int> e_try;  // > 0: faces per patch; < 0: balanced for -n stages
    if (auto_e && e_stages_req > 0) e_try = {-e_stages_req, 32, 16, 8};
    else if (auto_e) e_try = {-2, -3, 32, 16, 8};
    else e_try = {fpp_e};
    if (!quads_fit) e_try.clear();
    std::vector<char> v_src(nV, 0), e_src(nE, 0);
    for (int s = 0; s < X->n_src_er; ++s) v_src[X->src_er_vertex[s]] = 1;
    for (int s = 0; s < X->n_src_et; ++s) e_src[X->src_et_edge[s]] = 1;
    for (const int c : e_try) {
      const int stages_wanted = c < 0 ? -c : 2;
      // bridged gaps add rows the balance does not count: leave them room
      const int margin = 97 - 3 * e_copy_gap;
      Own o = c < 0 ? ownership_bounds(balanced_e_bounds(stage_budget / stages_wanted * margin / 100, plasma, (int)sizeof(real)))
                    : ownership(c);
      Slots sl;
      if (!build_slots(o.vlist, sl)) break;
      PipeTables t;
      const bool ok = build_pipe_e<real>(t, o.n, o.vptr, o.vlist, o.eptr, lr, SW, sl.edge, sl.face, sl.coef, sl.wc,
                                         inv_phi, tn, plasma, Pn, Pm, v_src, e_src, locA, locB,
                                         stage_budget / stages_wanted, e_copy_gap);
      if (ok && stages_wanted * t.stage_bytes <= stage_budget) {
        P->pipe_e_ok = true;
        fpp_e = c > 0 ? c : 0;
        oe = std::move(o);
        slots = std::move(sl);
        te_tab = std::move(t);
        break;
      }
    }
    if (P->pipe_h_ok && !descriptors_valid(th_tab, (int)sizeof(real), Pn, Pm, X->si_terms, nV, nE, nF, S))
      P->pipe_h_ok = false;
    if (P->pipe_e_ok && !descriptors_valid(te_tab, (int)sizeof(real), Pn, Pm, 0, nV, nE, nF, plasma ? 1 : 0))
      P->pipe_e_ok = false;
    P->kh_stage = th_tab.stage_bytes;
    P->ke_stage = te_tab.stage_bytes;
    auto patch_costs = [](const PipeTables& t) {
      std::vector<float> c(t.dptr.size() - 1, 0.f);
      for (size_t q = 0; q + 1 < t.dptr.size(); ++q)
        for (int d = t.dptr[q]; d < t.dptr[q + 1]; ++d) c[q] += (float)t.desc[d].w;
      return c;
    };
    if (P->pipe_h_ok) P->kh_cost = patch_costs(th_tab);
    if (P->pipe_e_ok) P->ke_cost = patch_costs(te_tab);
    if (P->pipe_h_ok) {
      UP(th_tab.dptr, dptr_h);
      UP(th_tab.desc, desc_h);
      UP(th_tab.tab, tab_h);
    }
    if (P->pipe_e_ok) {
      UP(te_tab.dptr, dptr_e);
      UP(te_tab.desc, desc_e);
      UP(te_tab.tab, tab_e);
    }
  }
  if (P->fused_pipe) {
    UP(tf_tab.dptr, dptr_e);
    UP(tf_tab.desc, desc_e);
    UP(tf_tab.tab, tab_e);
  }
  P->n_patches = oh.n;
  P->n_patches_e = oe.n;
  UP(oh.eptr, eptr_h);
  UP(oe.eptr, eptr_e);
  UP(oe.vptr, vptr);
  UP(oe.vlist, vlist);
  UP(slots.edge, ps_edge);
  UP(slots.coef, ps_coef);
  if (plasma) {
    UP(slots.face, ps_face);
    UP(slots.wc, ps_wc);
  }
#undef UP

  // ---- record ----
  R.nV = nV;
  R.nE = nE;
  R.nF = nF;
  R.L = L;
  R.Pn = Pn;
  R.Pm = Pm;
  R.n_patches_h = oh.n;
  R.fpp_h = fpp;
  R.n_patches_e = oe.n;
  R.fpp_e = fpp_e;
  R.full = G->full_spherical ? 1 : 0;
  R.si_terms = X->si_terms;
  R.n_species = X->plasma_species;
  R.plasma_full = X->plasma_rows == nF && nF != 1 ? 1 : 0;
  R.magnetized = X->plasma_magnetized ? 1 : 0;
  R.coef_full = X->coef_rows_er != 1 ? 1 : 0;
  R.plasma_local = local ? 1 : 0;
  R.n_src_er = X->n_src_er;
  R.n_src_et = X->n_src_et;
  R.maxdeg = MD;
  R.slot_width = SW;
  R.layer_reals = layer_reals(Pn, Pm, R.coef_full, X->plasma_species, R.plasma_full, R.magnetized, X->si_terms);
  P->smem_bytes = (size_t)R.layer_reals * sizeof(real);
  if (P->smem_bytes > 200 * 1024) return fail(IFDTD_ERR_UNSUPPORTED, "radial grid too fine for the shared per-layer rows");
  {
    // pipelined kernels: per-layer rows + n_stages ring stages in dynamic shared memory
    if (pipe::layer_block_bytes(R.layer_reals, (int)sizeof(real)) != layer_block)
      return fail(IFDTD_ERR_UNSUPPORTED, "inconsistent shared per-layer rows");
    auto stages = [&](bool ok, int stage) {
      return ok && stage > 0 ? std::min(pipe::kMaxStages, stage_budget / stage) : 0;
    };
    P->kh_stages = stages(P->pipe_h_ok, P->kh_stage);
    P->ke_stages = stages(P->pipe_e_ok, P->ke_stage);
    P->kh_smem = (size_t)layer_block + (size_t)P->kh_stages * P->kh_stage;
    P->ke_smem = (size_t)layer_block + (size_t)P->ke_stages * P->ke_stage;
    auto pick = [&](int n_stages) { return staging == 1 ? 1 : (n_stages >= 2 ? 2 : (staging >= 2 ? 0 : 1)); };
    P->h_mode = pick(P->kh_stages);
    P->e_mode = pick(P->ke_stages);
    if (P->h_mode == 0 || P->e_mode == 0)
      return fail(IFDTD_ERR_UNSUPPORTED, "pipelined kernels need at least two patch stages in shared memory");
    if ((P->h_mode == 1 || P->e_mode == 1) && threads > 256)
      return fail(IFDTD_ERR_ARGUMENT, "direct kernels take at most 256 threads per CTA");
    if (auto_threads && P->h_mode == 2 && P->e_mode == 2) threads = pipe::kMaxThreads - 32 * producers;
    P->threads = threads;
    // E-phase compute threads: as given; automatic with automatic threads: the
    // pipelined CTA's 384 less the E producer warps; otherwise as threads
    P->e_threads = e_threads_req > 0 ? e_threads_req
                   : (auto_threads && P->h_mode == 2 && P->e_mode == 2) ? pipe::kMaxThreads - 32 * e_producers
                                                                        : threads;
    if (P->e_mode == 2 && P->e_threads + 32 * e_producers > pipe::kMaxThreads &&
        (e_threads_req == 0 || P->pipe_copy != 0))
      return fail(IFDTD_ERR_ARGUMENT, "threads + 32 * E producer warps must not exceed 384");
    // rows on 8-lane boundaries only while a rounded-up row still fits the
    // compute threads of both phases (otherwise the rows stay packed)
    const int wide = std::max((Pn / (int)(16 / sizeof(real)) + 7) & ~7, (Pm / (int)(16 / sizeof(real)) + 7) & ~7);
    P->lanes = lane_layout == 2 && wide <= std::min(threads, P->e_threads) ? 1 : 0;
  }
  {
    void* st = nullptr;
    cudaError_t e = A.alloc(sizeof(int), &st);
    if (e != cudaSuccess) return fail(IFDTD_ERR_CUDA, "allocation of the status word failed");
    CUDA_TRY(cudaMemset(st, 0, sizeof(int)));
    P->d_status = (int*)st;
    R.status = (int*)st;
  }
  R.dtmu = (real)(G->time_step_s / 1.256637062120e-6);
  {
    void* cur = nullptr;
    cudaError_t e = A.alloc(std::max(P->chunk, 1) * sizeof(double), &cur);
    if (e != cudaSuccess) return fail(IFDTD_ERR_CUDA, "allocation of current staging failed");
    P->d_cur = (double*)cur;
    R.cur = P->d_cur;
  }
  P->h_rec.resize(sizeof(Rec<real>));
  std::memcpy(P->h_rec.data(), &R, sizeof(R));
  {
    cudaError_t e = A.alloc(sizeof(Rec<real>), &P->d_rec);
    if (e != cudaSuccess) return fail(IFDTD_ERR_CUDA, "allocation of launch record failed");
    CUDA_TRY(cudaMemcpy(P->d_rec, &R, sizeof(R), cudaMemcpyHostToDevice));
  }
  if (P->fused) {
    // the record of the second field copy: the plan's record with the four field pointers moved
    Rec<real> rb = R;
    rb.er = (real*)P->fb[0];
    rb.et = (real*)P->fb[1];
    rb.hr = (real*)P->fb[2];
    rb.ht = (real*)P->fb[3];
    cudaError_t e = A.alloc(sizeof(Rec<real>), &P->d_rec_b);
    if (e != cudaSuccess) return fail(IFDTD_ERR_CUDA, "allocation of the second launch record failed");
    CUDA_TRY(cudaMemcpy(P->d_rec_b, &rb, sizeof(rb), cudaMemcpyHostToDevice));
  }
  CUDA_TRY(cudaStreamCreateWithFlags(&P->capture_stream, cudaStreamNonBlocking));
  return IFDTD_OK;
}

// Refresh the state pointers in the device record when they changed.
template <typename real>
int bind_state(ifdtd_plan* P, const ifdtd_state* st, cudaStream_t stream) {
  if (!st || !st->er || !st->et || !st->hr || !st->ht) return fail(IFDTD_ERR_ARGUMENT, "state pointers missing");
  if (P->T > 0 && !st->si_memory) return fail(IFDTD_ERR_ARGUMENT, "surface impedance memory missing");
  for (int s = 0; s < P->S; ++s)
    if (!st->plasma_current[s]) return fail(IFDTD_ERR_ARGUMENT, "plasma current missing");
  if (P->have_state && std::memcmp(&P->last_state, st, sizeof(*st)) == 0) return IFDTD_OK;
  Rec<real>* R = reinterpret_cast<Rec<real>*>(P->h_rec.data());
  R->er = (real*)st->er;
  R->et = (real*)st->et;
  R->hr = (real*)st->hr;
  R->ht = (real*)st->ht;
  R->si_mem = (real*)st->si_memory;
  for (int s = 0; s < kMaxSpecies; ++s) R->J[s] = (real*)st->plasma_current[s];
  // pageable source: the runtime stages it before returning, so h_rec may change afterwards
  CUDA_TRY(cudaMemcpyAsync(P->d_rec, P->h_rec.data(), sizeof(Rec<real>), cudaMemcpyHostToDevice, stream));
  P->last_state = *st;
  P->have_state = true;
  return IFDTD_OK;
}

// Dynamic shared memory above 48 KiB is opted into per kernel function.  The
// limit is only ever raised: plans and batch groups that launch the same
// instantiation with smaller stages (and graphs captured for them) stay valid.
template <typename K>
cudaError_t allow_smem(K kernel, size_t bytes) {
  if (bytes <= 48 * 1024) return cudaSuccess;
  cudaFuncAttributes attr;
  cudaError_t e = cudaFuncGetAttributes(&attr, kernel);
  if (e != cudaSuccess) return e;
  if ((size_t)attr.maxDynamicSharedSizeBytes >= bytes) return cudaSuccess;
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// Persistent grid: SM count x resident CTAs (from the occupancy calculator).
template <typename K>
cudaError_t persistent_grid(ifdtd_plan* P, K kernel, int threads, size_t smem, int n_patches, int* grid) {
  if (*grid > 0) return cudaSuccess;
  int per_sm = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  *grid = std::max(1, std::min(n_patches, P->sm_count * per_sm));
  return cudaSuccess;
}

template <typename real, bool PL>
cudaError_t launch_kh_t(ifdtd_plan* P, const Rec<real>* rec, cudaStream_t st) {
  if (P->h_mode == 2) {
    auto k = P->pipe_copy == 0 ? pipe::kh_tma<real, PL, 0> : pipe::kh_tma<real, PL, 1>;
    const int threads = P->threads + 32 * P->producers;
    cudaError_t e = allow_smem(k, P->kh_smem);
    if (e == cudaSuccess) e = persistent_grid(P, k, threads, P->kh_smem, P->n_patches, &P->kh_grid);
    if (e != cudaSuccess) return e;
    k<<<P->kh_grid, threads, P->kh_smem, st>>>(rec, P->kh_stage, P->kh_stages, P->producers, P->lanes);
  } else {
    auto k = kh_kernel<real, PL>;
    cudaError_t e = allow_smem(k, P->smem_bytes);
    if (e != cudaSuccess) return e;
    k<<<P->n_patches, P->threads, P->smem_bytes, st>>>(rec, nullptr, 1);
  }
  return cudaGetLastError();
}

template <typename real, bool PL, int MD>
cudaError_t launch_ke_t(ifdtd_plan* P, const Rec<real>* rec, int istep, cudaStream_t st) {
  if (P->e_mode == 2) {
    const int threads = P->e_threads + 32 * P->e_producers;
    auto k = threads > pipe::kMaxThreads ? pipe::ke_tma<real, PL, MD, 0, pipe::kWideRegs>
             : P->pipe_copy == 0         ? pipe::ke_tma<real, PL, MD, 0, pipe::kMaxRegs>
                                         : pipe::ke_tma<real, PL, MD, 1, pipe::kMaxRegs>;
    cudaError_t e = allow_smem(k, P->ke_smem);
    if (e == cudaSuccess) e = persistent_grid(P, k, threads, P->ke_smem, P->n_patches_e, &P->ke_grid);
    if (e != cudaSuccess) return e;
    k<<<P->ke_grid, threads, P->ke_smem, st>>>(rec, P->ke_stage, P->ke_stages, P->e_producers, istep, P->lanes);
  } else {
    auto k = ke_kernel<real, PL, MD>;
    cudaError_t e = allow_smem(k, P->smem_bytes);
    if (e != cudaSuccess) return e;
    k<<<P->n_patches_e, P->threads, P->smem_bytes, st>>>(rec, nullptr, 1, istep);
  }
  return cudaGetLastError();
}

template <typename real>
cudaError_t launch_kh(ifdtd_plan* P, cudaStream_t st) {
  const Rec<real>* rec = (const Rec<real>*)P->d_rec;
  return P->plasma ? launch_kh_t<real, true>(P, rec, st) : launch_kh_t<real, false>(P, rec, st);
}

template <typename real>
cudaError_t launch_ke(ifdtd_plan* P, int istep, cudaStream_t st) {
  const Rec<real>* rec = (const Rec<real>*)P->d_rec;
  if (P->maxdeg == 6)
    return P->plasma ? launch_ke_t<real, true, 6>(P, rec, istep, st) : launch_ke_t<real, false, 6>(P, rec, istep, st);
  return P->plasma ? launch_ke_t<real, true, 12>(P, rec, istep, st) : launch_ke_t<real, false, 12>(P, rec, istep, st);
}

// One fused step: parity 0 reads the caller's arrays and writes the plan's
// second copy, parity 1 the reverse.
template <typename real>
cudaError_t launch_fused(ifdtd_plan* P, int istep, int parity, cudaStream_t st) {
  const Rec<real>* a = (const Rec<real>*)P->d_rec;
  const Rec<real>* b = (const Rec<real>*)P->d_rec_b;
  if (P->fused_pipe) {
    const int threads = P->kf_threads + 32 * P->kf_producers;
    auto k = P->maxdeg == 6 ? (P->pipe_copy == 0 ? pipe::kf_tma<real, 6, 0> : pipe::kf_tma<real, 6, 1>)
                            : (P->pipe_copy == 0 ? pipe::kf_tma<real, 12, 0> : pipe::kf_tma<real, 12, 1>);
    cudaError_t e = allow_smem(k, P->kf_smem);
    if (e == cudaSuccess) e = persistent_grid(P, k, threads, P->kf_smem, P->n_patches_e, &P->kf_grid);
    if (e != cudaSuccess) return e;
    k<<<P->kf_grid, threads, P->kf_smem, st>>>(parity ? b : a, parity ? a : b, P->kf_stage, P->kf_stages,
                                               P->kf_producers, istep, P->kf_lanes);
    return cudaGetLastError();
  }
  auto k = P->maxdeg == 6 ? fused_step_kernel<real, 6> : fused_step_kernel<real, 12>;
  cudaError_t e = allow_smem(k, P->fused_smem);
  if (e != cudaSuccess) return e;
  k<<<P->n_patches_e, P->threads, P->fused_smem, st>>>(parity ? b : a, parity ? a : b, P->fused_tab, istep);
  return cudaGetLastError();
}

template <typename real>
cudaError_t launch_step(ifdtd_plan* P, int istep, const ifdtd_probe* probe, int row, cudaStream_t st, int parity = 0) {
  const Rec<real>* rec = (const Rec<real>*)P->d_rec;
  cudaError_t e;
  if (P->fused) {
    e = launch_fused<real>(P, istep, parity, st);
    // the step's result is in the copy it wrote
    if (!parity) rec = (const Rec<real>*)P->d_rec_b;
  } else {
    e = launch_kh<real>(P, st);
    if (e == cudaSuccess) e = launch_ke<real>(P, istep, st);
  }
  if (e != cudaSuccess) return e;
  if (probe) {
    const int blocks = (probe->rows * 32 + 255) / 256;
    sample_rec_kernel<real><<<blocks, 256, 0, st>>>(rec, probe->kind, probe->rows, probe->width, probe->index,
                                                     probe->layer, probe->weight,
                                                     probe->staging + (size_t)row * probe->rows);
  }
  return cudaGetLastError();
}

// Face frames: the caller's Cartesian plasma currents turned into the plan's
// face frames before a call's first phase kernel (to_local 1) and back after
// its last (to_local 0), so the state between calls is Cartesian.  A call that
// fails in between leaves the currents in face frames (its results are invalid
// anyway).
template <typename real>
cudaError_t plasma_frames(const ifdtd_plan* P, const ifdtd_state* st, int to_local, cudaStream_t stream) {
  if (!P->plasma_local) return cudaSuccess;
  const size_t items = (size_t)P->nF * (size_t)(P->Pm / Lanes<real>::N);
  const int grid = (int)std::min<size_t>(std::max<size_t>((items + 255) / 256, 1), (size_t)P->sm_count * 8);
  for (int s = 0; s < P->S; ++s)
    plasma_frame_kernel<real><<<grid, 256, 0, stream>>>(static_cast<real*>(st->plasma_current[s]),
                                                        static_cast<const real*>(P->d_frame), P->nF, P->Pm, to_local);
  return cudaGetLastError();
}

template <typename real>
int run_steps(ifdtd_plan* P, const ifdtd_state* st, const double* currents, int n, const ifdtd_probe* probe,
              double* out_rows, cudaStream_t stream) {
  int rc = bind_state<real>(P, st, stream);
  if (rc) return rc;
  if (n <= 0) return IFDTD_OK;
  CUDA_TRY(plasma_frames<real>(P, st, 1, stream));
  // NVTX range over the host-side enqueue of these steps (visible to profilers)
  struct Range {
    explicit Range(const char* name) { nvtxRangePushA(name); }
    ~Range() { nvtxRangePop(); }
  } range(probe ? "ifdtd_step_sampled" : "ifdtd_step");
  const int cap = std::max(P->chunk, 1);
  int parity = 0;  // fused step: 1 while the state is in the plan's second copy
  for (int s0 = 0; s0 < n; s0 += cap) {
    const int c = std::min(cap, n - s0);
    if (currents)
      CUDA_TRY(cudaMemcpyAsync(P->d_cur, currents + s0, c * sizeof(double), cudaMemcpyDeviceToDevice, stream));
    else
      CUDA_TRY(cudaMemsetAsync(P->d_cur, 0, c * sizeof(double), stream));
    if (P->chunk > 0 && c == P->chunk) {
      cudaGraphExec_t exec = nullptr;
      for (auto& g : P->graphs)
        if (g.chunk == c && g.probe == probe) exec = g.exec;
      if (!exec) {
        cudaGraph_t graph;
        CUDA_TRY(cudaStreamBeginCapture(P->capture_stream, cudaStreamCaptureModeThreadLocal));
        cudaError_t le = cudaSuccess;
        // an even chunk (fused plans) starts and ends in the caller's arrays
        for (int i = 0; i < c && le == cudaSuccess; ++i)
          le = launch_step<real>(P, i, probe, i, P->capture_stream, P->fused ? (i & 1) : 0);
        cudaError_t ce = cudaStreamEndCapture(P->capture_stream, &graph);
        if (le != cudaSuccess) {
          if (ce == cudaSuccess) cudaGraphDestroy(graph);  // the partial capture is not kept
          return fail(IFDTD_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(le));
        }
        if (ce != cudaSuccess) return fail(IFDTD_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
        cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ie != cudaSuccess) return fail(IFDTD_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ie));
        P->graphs.push_back({c, probe, exec});
      }
      CUDA_TRY(cudaGraphLaunch(exec, stream));
    } else {
      for (int i = 0; i < c; ++i) {
        cudaError_t e = launch_step<real>(P, i, probe, i, stream, parity);
        if (e != cudaSuccess) return fail(IFDTD_ERR_CUDA, std::string("step launch: ") + cudaGetErrorString(e));
        if (P->fused) parity ^= 1;
      }
    }
    if (probe && out_rows)
      CUDA_TRY(cudaMemcpyAsync(out_rows + (size_t)s0 * probe->rows, probe->staging,
                               (size_t)c * probe->rows * sizeof(double), cudaMemcpyDeviceToDevice, stream));
  }
  if (parity) {
    // an odd number of fused steps ended in the second copy: move it to the caller's arrays
    void* const dst[4] = {st->er, st->et, st->hr, st->ht};
    for (int i = 0; i < 4; ++i)
      CUDA_TRY(cudaMemcpyAsync(dst[i], P->fb[i], P->fb_bytes[i], cudaMemcpyDeviceToDevice, stream));
  }
  CUDA_TRY(plasma_frames<real>(P, st, 0, stream));
  return IFDTD_OK;
}

struct DeviceGuard {
  int previous = -1;
  explicit DeviceGuard(int device) {
    if (cudaGetDevice(&previous) == cudaSuccess && previous != device) cudaSetDevice(device);
    else previous = -1;
  }
  ~DeviceGuard() {
    if (previous >= 0) cudaSetDevice(previous);
  }
};

int grid_for(size_t n) {
  size_t b = (n + 255) / 256;
  return (int)std::min<size_t>(std::max<size_t>(b, 1), 148 * 16);
}

}  // namespace

// ---------------------------------------------------------------------------
// Ensembles: member plans advanced together.  Members whose two phases both
// run on the pipeline are grouped by kernel template (precision is the
// batch's; plasma, vertex slot width, copy engine, threads and producer warps
// per group) and every group takes one batched launch per phase: CTAs walk
// cost-balanced ranges of the members' concatenated patch lists.  Other
// members launch on their own inside the same step.  Receivers of all members
// are sampled by one launch per step.
// ---------------------------------------------------------------------------
struct BatchGroup {
  // fused: members on the fused step (pipe::kf_tma_batch; threads, producers
  // and lanes are then the fused kernel's)
  int fused = 0, plasma = 0, maxdeg = 6, copy = 0, threads = 0, producers = 2, lanes = 0, e_threads = 0, e_producers = 2;
  std::vector<int> members;
  size_t kh_smem = 0, ke_smem = 0, kf_smem = 0;
  int kh_grid = 0, ke_grid = 0, kf_grid = 0;
  const int4* segs_f = nullptr;
  const int* sptr_f = nullptr;
  const int4* segs_h = nullptr;
  const int* sptr_h = nullptr;
  const int4* segs_e = nullptr;
  const int* sptr_e = nullptr;
};

struct ifdtd_batch {
  int device = 0, dtype = 4, n = 0, chunk = 32;
  std::vector<ifdtd_plan*> plans;
  std::vector<int> solo;  // members with a direct-kernel phase
  std::vector<BatchGroup> groups;
  DeviceArena arena;
  void* d_recs = nullptr;  // one record per member: bound fields, currents from d_cur
  std::vector<unsigned char> h_recs;
  // fused-step members: their records pointed at the plans' second field
  // copies (other members' records as in d_recs), and the ring table
  bool any_fused = false;
  void* d_recs_b = nullptr;
  std::vector<unsigned char> h_recs_b;
  const int2* d_ring_f = nullptr;
  size_t rec_bytes = 0;
  double* d_cur = nullptr;  // (n, chunk) step currents
  const int2* d_ring_h = nullptr;
  const int2* d_ring_e = nullptr;
  // sampled steps: probe table, row map and (chunk, rows) staging; they grow
  // on demand and every captured graph is dropped when they move
  void* d_refs = nullptr;
  void* d_rowmap = nullptr;
  double* d_stage = nullptr;
  int cap_refs = 0, cap_rows = 0;
  std::vector<ifdtd_state> last;
  bool have_state = false;
  cudaStream_t capture_stream = nullptr;
  struct Graph {
    int chunk, rows;
    cudaGraphExec_t exec;
  };
  std::vector<Graph> graphs;
  std::string failed;  // the launch that failed last (error messages)
  void drop_graphs() {
    for (auto& g : graphs) cudaGraphExecDestroy(g.exec);
    graphs.clear();
  }
  ~ifdtd_batch() {
    drop_graphs();
    if (capture_stream) cudaStreamDestroy(capture_stream);
    cudaFree(d_refs);
    cudaFree(d_rowmap);
    cudaFree(d_stage);
  }
};

namespace {

// Cost-balanced contiguous ranges of the members' concatenated patch lists,
// one per CTA, cut at member boundaries into segments {member, first patch,
// end patch, 0}; CTA b owns segs[sptr[b]] .. segs[sptr[b + 1] - 1].  A patch
// goes to the CTA in whose share its cost midpoint falls; the last CTA takes
// the rest.
void split_patches(const std::vector<int>& members, const std::vector<const std::vector<float>*>& cost, int grid,
                   std::vector<int4>& segs, std::vector<int>& sptr) {
  double total = 0.0;
  for (const auto* c : cost)
    for (const float x : *c) total += std::max(x, 1.0f);
  segs.clear();
  sptr.assign(1, 0);
  size_t mi = 0;
  int p = 0;
  double acc = 0.0;
  for (int b = 0; b < grid; ++b) {
    const double end = total * (b + 1) / grid;
    while (mi < members.size()) {
      const std::vector<float>& cv = *cost[mi];
      if (p >= (int)cv.size()) {
        ++mi;
        p = 0;
        continue;
      }
      const double w = std::max(cv[p], 1.0f);
      if (b + 1 < grid && acc + 0.5 * w > end) break;
      if ((int)segs.size() > sptr.back() && segs.back().x == members[mi] && segs.back().z == p)
        segs.back().z = p + 1;
      else
        segs.push_back(make_int4(members[mi], p, p + 1, 0));
      acc += w;
      ++p;
    }
    sptr.push_back((int)segs.size());
  }
}

template <typename real>
auto batch_kh_kernel(const BatchGroup& g) {
  using namespace pipe;
  if (g.plasma) return g.copy ? kh_tma_batch<real, true, 1> : kh_tma_batch<real, true, 0>;
  return g.copy ? kh_tma_batch<real, false, 1> : kh_tma_batch<real, false, 0>;
}

template <typename real>
auto batch_ke_kernel(const BatchGroup& g) {
  using namespace pipe;
  const bool wide = g.e_threads + 32 * g.e_producers > kMaxThreads;
  if (g.plasma) {
    if (g.maxdeg == 6)
      return wide ? ke_tma_batch<real, true, 6, 0, kWideRegs>
                  : g.copy ? ke_tma_batch<real, true, 6, 1, kMaxRegs> : ke_tma_batch<real, true, 6, 0, kMaxRegs>;
    return wide ? ke_tma_batch<real, true, 12, 0, kWideRegs>
                : g.copy ? ke_tma_batch<real, true, 12, 1, kMaxRegs> : ke_tma_batch<real, true, 12, 0, kMaxRegs>;
  }
  if (g.maxdeg == 6)
    return wide ? ke_tma_batch<real, false, 6, 0, kWideRegs>
                : g.copy ? ke_tma_batch<real, false, 6, 1, kMaxRegs> : ke_tma_batch<real, false, 6, 0, kMaxRegs>;
  return wide ? ke_tma_batch<real, false, 12, 0, kWideRegs>
              : g.copy ? ke_tma_batch<real, false, 12, 1, kMaxRegs> : ke_tma_batch<real, false, 12, 0, kMaxRegs>;
}

template <typename real>
auto batch_kf_kernel(const BatchGroup& g) {
  using namespace pipe;
  if (g.maxdeg == 6) return g.copy ? kf_tma_batch<real, 6, 1> : kf_tma_batch<real, 6, 0>;
  return g.copy ? kf_tma_batch<real, 12, 1> : kf_tma_batch<real, 12, 0>;
}

template <typename K>
cudaError_t batch_grid(K kernel, int threads, size_t smem, int sm_count, int n_patches, int* grid) {
  cudaError_t e = allow_smem(kernel, smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  *grid = std::max(1, std::min(n_patches, sm_count * per_sm));
  return cudaSuccess;
}

template <typename real>
int batch_build(ifdtd_batch* B) {
  B->rec_bytes = sizeof(Rec<real>);
  for (int i = 0; i < B->n; ++i) {
    ifdtd_plan* P = B->plans[i];
    BatchGroup key;
    if (P->fused) {
      if (!P->fused_pipe) return fail(IFDTD_ERR_UNSUPPORTED, "a fused-step plan on direct gathers cannot join a batch");
      key.fused = 1;
      key.maxdeg = P->maxdeg;
      key.copy = P->pipe_copy;
      key.threads = P->kf_threads;
      key.producers = P->kf_producers;
      key.lanes = P->kf_lanes;
      key.e_threads = key.e_producers = 0;
      B->any_fused = true;
    } else if (P->h_mode != 2 || P->e_mode != 2) {
      B->solo.push_back(i);
      continue;
    } else {
      key.plasma = P->plasma ? 1 : 0;
      key.maxdeg = P->maxdeg;
      key.copy = P->pipe_copy;
      key.threads = P->threads;
      key.producers = P->producers;
      key.lanes = P->lanes;
      key.e_threads = P->e_threads;
      key.e_producers = P->e_producers;
    }
    BatchGroup* g = nullptr;
    for (auto& x : B->groups)
      if (x.fused == key.fused && x.plasma == key.plasma && x.maxdeg == key.maxdeg && x.copy == key.copy &&
          x.threads == key.threads && x.producers == key.producers && x.lanes == key.lanes &&
          x.e_threads == key.e_threads && x.e_producers == key.e_producers)
        g = &x;
    if (!g) {
      B->groups.push_back(key);
      g = &B->groups.back();
    }
    g->members.push_back(i);
  }
  std::vector<int2> ring_h(B->n, make_int2(0, 0)), ring_e(B->n, make_int2(0, 0)), ring_f(B->n, make_int2(0, 0));
  for (const auto& g : B->groups)
    for (const int i : g.members) {
      const ifdtd_plan* P = B->plans[i];
      ring_h[i] = make_int2(P->kh_stage, P->kh_stages);
      ring_e[i] = make_int2(P->ke_stage, P->ke_stages);
      ring_f[i] = make_int2(P->kf_stage, P->kf_stages);
    }
  if (B->arena.upload(ring_h, &B->d_ring_h) != cudaSuccess || B->arena.upload(ring_e, &B->d_ring_e) != cudaSuccess ||
      B->arena.upload(ring_f, &B->d_ring_f) != cudaSuccess)
    return fail(IFDTD_ERR_CUDA, "upload of batch ring table failed");
  const int sm_count = B->plans[0]->sm_count;
  for (auto& g : B->groups) {
    if (g.fused) {
      int nf = 0;
      std::vector<const std::vector<float>*> cf;
      for (const int i : g.members) {
        const ifdtd_plan* P = B->plans[i];
        g.kf_smem = std::max(g.kf_smem, P->kf_smem);
        nf += P->n_patches_e;
        cf.push_back(&P->kf_cost);
      }
      cudaError_t e = batch_grid(batch_kf_kernel<real>(g), g.threads + 32 * g.producers, g.kf_smem, sm_count, nf, &g.kf_grid);
      if (e != cudaSuccess) return fail(IFDTD_ERR_CUDA, std::string("batched launch shape: ") + cudaGetErrorString(e));
      std::vector<int4> segs;
      std::vector<int> sptr;
      split_patches(g.members, cf, g.kf_grid, segs, sptr);
      if (B->arena.upload(segs, &g.segs_f) != cudaSuccess || B->arena.upload(sptr, &g.sptr_f) != cudaSuccess)
        return fail(IFDTD_ERR_CUDA, "upload of batch segments failed");
      continue;
    }
    int nh = 0, ne = 0;
    std::vector<const std::vector<float>*> ch, ce;
    for (const int i : g.members) {
      const ifdtd_plan* P = B->plans[i];
      g.kh_smem = std::max(g.kh_smem, P->kh_smem);
      g.ke_smem = std::max(g.ke_smem, P->ke_smem);
      nh += P->n_patches;
      ne += P->n_patches_e;
      ch.push_back(&P->kh_cost);
      ce.push_back(&P->ke_cost);
    }
    const int threads = g.threads + 32 * g.producers, e_threads = g.e_threads + 32 * g.e_producers;
    cudaError_t e = batch_grid(batch_kh_kernel<real>(g), threads, g.kh_smem, sm_count, nh, &g.kh_grid);
    if (e == cudaSuccess) e = batch_grid(batch_ke_kernel<real>(g), e_threads, g.ke_smem, sm_count, ne, &g.ke_grid);
    if (e != cudaSuccess) return fail(IFDTD_ERR_CUDA, std::string("batched launch shape: ") + cudaGetErrorString(e));
    std::vector<int4> segs;
    std::vector<int> sptr;
    split_patches(g.members, ch, g.kh_grid, segs, sptr);
    if (B->arena.upload(segs, &g.segs_h) != cudaSuccess || B->arena.upload(sptr, &g.sptr_h) != cudaSuccess)
      return fail(IFDTD_ERR_CUDA, "upload of batch segments failed");
    split_patches(g.members, ce, g.ke_grid, segs, sptr);
    if (B->arena.upload(segs, &g.segs_e) != cudaSuccess || B->arena.upload(sptr, &g.sptr_e) != cudaSuccess)
      return fail(IFDTD_ERR_CUDA, "upload of batch segments failed");
  }
  void* cur = nullptr;
  void* recs = nullptr;
  if (B->arena.alloc((size_t)B->n * B->chunk * sizeof(double), &cur) != cudaSuccess ||
      B->arena.alloc((size_t)B->n * B->rec_bytes, &recs) != cudaSuccess)
    return fail(IFDTD_ERR_CUDA, "allocation of batch records failed");
  B->d_cur = (double*)cur;
  B->d_recs = recs;
  B->h_recs.assign((size_t)B->n * B->rec_bytes, 0);
  for (int i = 0; i < B->n; ++i) {
    std::memcpy(B->h_recs.data() + (size_t)i * B->rec_bytes, B->plans[i]->h_rec.data(), B->rec_bytes);
    reinterpret_cast<Rec<real>*>(B->h_recs.data() + (size_t)i * B->rec_bytes)->cur = B->d_cur + (size_t)i * B->chunk;
  }
  if (B->any_fused && B->arena.alloc((size_t)B->n * B->rec_bytes, &B->d_recs_b) != cudaSuccess)
    return fail(IFDTD_ERR_CUDA, "allocation of batch records failed");
  CUDA_TRY(cudaStreamCreateWithFlags(&B->capture_stream, cudaStreamNonBlocking));
  return IFDTD_OK;
}

// parity (fused-step members): 0 reads the caller's arrays and writes the
// plans' second copies, 1 the reverse.
template <typename real>
cudaError_t batch_launch_step(ifdtd_batch* B, int istep, int rows, int step_row, cudaStream_t st, int parity = 0) {
  const Rec<real>* recs = (const Rec<real>*)B->d_recs;
  const Rec<real>* recs_b = (const Rec<real>*)B->d_recs_b;
  cudaError_t e = cudaSuccess;
  // every launch is checked at once, so a failure reports its own error
  // rather than the invalidated capture it leaves behind
  for (size_t q = 0; q < B->groups.size() && e == cudaSuccess; ++q) {
    const BatchGroup& g = B->groups[q];
    if (!g.fused) continue;
    auto k = batch_kf_kernel<real>(g);
    k<<<g.kf_grid, g.threads + 32 * g.producers, g.kf_smem, st>>>(parity ? recs_b : recs, parity ? recs : recs_b,
                                                                   g.segs_f, g.sptr_f, B->d_ring_f, g.producers, istep,
                                                                   g.lanes);
    e = cudaGetLastError();
    if (e != cudaSuccess) B->failed = "kf_tma_batch of group " + std::to_string(q);
  }
  for (size_t q = 0; q < B->groups.size() && e == cudaSuccess; ++q) {
    const BatchGroup& g = B->groups[q];
    if (g.fused) continue;
    auto k = batch_kh_kernel<real>(g);
    k<<<g.kh_grid, g.threads + 32 * g.producers, g.kh_smem, st>>>(recs, g.segs_h, g.sptr_h, B->d_ring_h, g.producers,
                                                                   g.lanes);
    e = cudaGetLastError();
    if (e != cudaSuccess) B->failed = "kh_tma_batch of group " + std::to_string(q);
  }
  for (size_t q = 0; q < B->solo.size() && e == cudaSuccess; ++q) {
    e = launch_kh<real>(B->plans[B->solo[q]], st);
    if (e != cudaSuccess) B->failed = "H phase of member " + std::to_string(B->solo[q]);
  }
  for (size_t q = 0; q < B->groups.size() && e == cudaSuccess; ++q) {
    const BatchGroup& g = B->groups[q];
    if (g.fused) continue;
    auto k = batch_ke_kernel<real>(g);
    k<<<g.ke_grid, g.e_threads + 32 * g.e_producers, g.ke_smem, st>>>(recs, g.segs_e, g.sptr_e, B->d_ring_e, g.e_producers,
                                                                   istep, g.lanes);
    e = cudaGetLastError();
    if (e != cudaSuccess) B->failed = "ke_tma_batch of group " + std::to_string(q);
  }
  for (size_t q = 0; q < B->solo.size() && e == cudaSuccess; ++q) {
    e = launch_ke<real>(B->plans[B->solo[q]], istep, st);
    if (e != cudaSuccess) B->failed = "E phase of member " + std::to_string(B->solo[q]);
  }
  if (rows > 0 && e == cudaSuccess) {
    // after a parity-0 step the fused members' state is in their second copies
    const Rec<real>* now = B->any_fused && !parity ? recs_b : recs;
    sample_batch_kernel<real><<<(rows * 32 + 255) / 256, 256, 0, st>>>(now, (const ProbeRef*)B->d_refs,
                                                                         (const int2*)B->d_rowmap, rows, step_row);
    e = cudaGetLastError();
    if (e != cudaSuccess) B->failed = "sample_batch_kernel";
  }
  return e;
}

template <typename real>
int run_batch(ifdtd_batch* B, const ifdtd_state* states, const double* currents, int n, ifdtd_probe* const* probes,
              double* const* out_rows, cudaStream_t stream) {
  for (int i = 0; i < B->n; ++i) {
    const ifdtd_plan* P = B->plans[i];
    const ifdtd_state& s = states[i];
    if (!s.er || !s.et || !s.hr || !s.ht) return fail(IFDTD_ERR_ARGUMENT, "state pointers missing");
    if (P->T > 0 && !s.si_memory) return fail(IFDTD_ERR_ARGUMENT, "surface impedance memory missing");
    for (int k = 0; k < P->S; ++k)
      if (!s.plasma_current[k]) return fail(IFDTD_ERR_ARGUMENT, "plasma current missing");
  }
  for (const int i : B->solo) {
    const int rc = bind_state<real>(B->plans[i], &states[i], stream);
    if (rc) return rc;
  }
  if (!B->have_state || std::memcmp(B->last.data(), states, (size_t)B->n * sizeof(ifdtd_state)) != 0) {
    for (int i = 0; i < B->n; ++i) {
      Rec<real>* R = reinterpret_cast<Rec<real>*>(B->h_recs.data() + (size_t)i * B->rec_bytes);
      const ifdtd_state& s = states[i];
      R->er = (real*)s.er;
      R->et = (real*)s.et;
      R->hr = (real*)s.hr;
      R->ht = (real*)s.ht;
      R->si_mem = (real*)s.si_memory;
      for (int k = 0; k < kMaxSpecies; ++k) R->J[k] = (real*)s.plasma_current[k];
    }
    // pageable source: the runtime stages it before returning
    CUDA_TRY(cudaMemcpyAsync(B->d_recs, B->h_recs.data(), B->h_recs.size(), cudaMemcpyHostToDevice, stream));
    if (B->any_fused) {
      B->h_recs_b = B->h_recs;
      for (int i = 0; i < B->n; ++i) {
        const ifdtd_plan* P = B->plans[i];
        if (!P->fused) continue;
        Rec<real>* R = reinterpret_cast<Rec<real>*>(B->h_recs_b.data() + (size_t)i * B->rec_bytes);
        R->er = (real*)P->fb[0];
        R->et = (real*)P->fb[1];
        R->hr = (real*)P->fb[2];
        R->ht = (real*)P->fb[3];
      }
      CUDA_TRY(cudaMemcpyAsync(B->d_recs_b, B->h_recs_b.data(), B->h_recs_b.size(), cudaMemcpyHostToDevice, stream));
    }
    B->last.assign(states, states + B->n);
    B->have_state = true;
  }
  // receiver rows of every probed member, in member order
  int rows = 0;
  std::vector<ProbeRef> refs;
  std::vector<int2> rowmap;
  std::vector<int> offset(B->n, -1);
  if (probes)
    for (int i = 0; i < B->n; ++i) {
      const ifdtd_probe* p = probes[i];
      if (!p) continue;
      if (p->plan != B->plans[i]) return fail(IFDTD_ERR_ARGUMENT, "probe belongs to another plan");
      if (!out_rows || !out_rows[i]) return fail(IFDTD_ERR_ARGUMENT, "output rows missing for a probed member");
      offset[i] = rows;
      for (int r = 0; r < p->rows; ++r) rowmap.push_back(make_int2((int)refs.size(), r));
      refs.push_back(ProbeRef{i, p->kind, p->rows, p->width, p->index, p->layer, p->weight, nullptr});
      rows += p->rows;
    }
  if (n <= 0) return IFDTD_OK;
  for (int i = 0; i < B->n; ++i) CUDA_TRY(plasma_frames<real>(B->plans[i], &states[i], 1, stream));
  if (rows > 0) {
    if ((int)refs.size() > B->cap_refs || rows > B->cap_rows) {
      CUDA_TRY(cudaStreamSynchronize(stream));
      B->drop_graphs();
      cudaFree(B->d_refs);
      cudaFree(B->d_rowmap);
      cudaFree(B->d_stage);
      B->d_refs = B->d_rowmap = nullptr;
      B->d_stage = nullptr;
      B->cap_refs = B->cap_rows = 0;
      CUDA_TRY(cudaMalloc(&B->d_refs, refs.size() * sizeof(ProbeRef)));
      CUDA_TRY(cudaMalloc(&B->d_rowmap, (size_t)rows * sizeof(int2)));
      CUDA_TRY(cudaMalloc((void**)&B->d_stage, (size_t)B->chunk * rows * sizeof(double)));
      B->cap_refs = (int)refs.size();
      B->cap_rows = rows;
    }
    for (auto& r : refs) r.staging = B->d_stage + offset[r.member];
    CUDA_TRY(cudaMemcpyAsync(B->d_refs, refs.data(), refs.size() * sizeof(ProbeRef), cudaMemcpyHostToDevice, stream));
    CUDA_TRY(cudaMemcpyAsync(B->d_rowmap, rowmap.data(), rowmap.size() * sizeof(int2), cudaMemcpyHostToDevice, stream));
  }
  struct Range {
    explicit Range(const char* name) { nvtxRangePushA(name); }
    ~Range() { nvtxRangePop(); }
  } range("ifdtd_batch_step");
  const int cap = std::max(B->chunk, 1);
  int parity = 0;  // fused-step members: 1 while their state is in the second copies
  for (int s0 = 0; s0 < n; s0 += cap) {
    const int c = std::min(cap, n - s0);
    if (currents) {
      CUDA_TRY(cudaMemcpy2DAsync(B->d_cur, (size_t)B->chunk * sizeof(double), currents + s0, (size_t)n * sizeof(double),
                                 (size_t)c * sizeof(double), B->n, cudaMemcpyDeviceToDevice, stream));
      for (const int i : B->solo)
        CUDA_TRY(cudaMemcpyAsync(B->plans[i]->d_cur, currents + (size_t)i * n + s0, c * sizeof(double),
                                 cudaMemcpyDeviceToDevice, stream));
    } else {
      CUDA_TRY(cudaMemsetAsync(B->d_cur, 0, (size_t)B->n * B->chunk * sizeof(double), stream));
      for (const int i : B->solo) CUDA_TRY(cudaMemsetAsync(B->plans[i]->d_cur, 0, c * sizeof(double), stream));
    }
    if (c == B->chunk) {
      cudaGraphExec_t exec = nullptr;
      for (auto& g : B->graphs)
        if (g.chunk == c && g.rows == rows) exec = g.exec;
      if (!exec) {
        cudaGraph_t graph;
        CUDA_TRY(cudaStreamBeginCapture(B->capture_stream, cudaStreamCaptureModeThreadLocal));
        cudaError_t le = cudaSuccess;
        // an even chunk (batches with fused-step members) starts and ends in the caller's arrays
        for (int i = 0; i < c && le == cudaSuccess; ++i)
          le = batch_launch_step<real>(B, i, rows, i, B->capture_stream, B->any_fused ? (i & 1) : 0);
        cudaError_t ce = cudaStreamEndCapture(B->capture_stream, &graph);
        if (le != cudaSuccess) {
          if (ce == cudaSuccess) cudaGraphDestroy(graph);  // the partial capture is not kept
          return fail(IFDTD_ERR_CUDA, "batch graph capture: " + B->failed + ": " + cudaGetErrorString(le));
        }
        if (ce != cudaSuccess) return fail(IFDTD_ERR_CUDA, std::string("batch graph capture: ") + cudaGetErrorString(ce));
        cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ie != cudaSuccess)
          return fail(IFDTD_ERR_CUDA, std::string("batch graph instantiate: ") + cudaGetErrorString(ie));
        B->graphs.push_back({c, rows, exec});
      }
      CUDA_TRY(cudaGraphLaunch(exec, stream));
    } else {
      for (int i = 0; i < c; ++i) {
        cudaError_t e = batch_launch_step<real>(B, i, rows, i, stream, parity);
        if (e != cudaSuccess) return fail(IFDTD_ERR_CUDA, "batch step launch: " + B->failed + ": " + cudaGetErrorString(e));
        if (B->any_fused) parity ^= 1;
      }
    }
    for (int i = 0; i < B->n; ++i) {
      if (offset[i] < 0) continue;
      const int r = probes[i]->rows;
      CUDA_TRY(cudaMemcpy2DAsync(out_rows[i] + (size_t)s0 * r, (size_t)r * sizeof(double), B->d_stage + offset[i],
                                 (size_t)rows * sizeof(double), (size_t)r * sizeof(double), c, cudaMemcpyDeviceToDevice,
                                 stream));
    }
  }
  if (parity) {
    // an odd number of steps left the fused members in their second copies
    for (int i = 0; i < B->n; ++i) {
      const ifdtd_plan* P = B->plans[i];
      if (!P->fused) continue;
      void* const dst[4] = {states[i].er, states[i].et, states[i].hr, states[i].ht};
      for (int k = 0; k < 4; ++k)
        CUDA_TRY(cudaMemcpyAsync(dst[k], P->fb[k], P->fb_bytes[k], cudaMemcpyDeviceToDevice, stream));
    }
  }
  for (int i = 0; i < B->n; ++i) CUDA_TRY(plasma_frames<real>(B->plans[i], &states[i], 0, stream));
  return IFDTD_OK;
}

}  // namespace

extern "C" {

int32_t ifdtd_version(void) { return 10000; }

int32_t ifdtd_last_error(char* buffer, size_t size) {
  if (!buffer || size == 0) return IFDTD_ERR_ARGUMENT;
  std::snprintf(buffer, size, "%s", g_last_error.c_str());
  return IFDTD_OK;
}

int32_t ifdtd_device_count(int32_t* count) {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (count) *count = (e == cudaSuccess) ? n : 0;
  if (e != cudaSuccess) return fail(IFDTD_ERR_UNSUPPORTED, cudaGetErrorString(e));
  return IFDTD_OK;
}

int32_t ifdtd_plan_create(const ifdtd_mesh_desc* mesh, const ifdtd_grid_desc* grid, const ifdtd_physics_desc* physics,
                          const ifdtd_tuning* tuning, int32_t dtype_bytes, int32_t device, ifdtd_plan** out) {
  if (!out || !mesh || !grid || !physics) return fail(IFDTD_ERR_ARGUMENT, "null argument");
  *out = nullptr;
  if (dtype_bytes != 4 && dtype_bytes != 8) return fail(IFDTD_ERR_ARGUMENT, "dtype must be 4 or 8 bytes");
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return fail(IFDTD_ERR_UNSUPPORTED, "no CUDA device");
  if (device < 0 || device >= n) return fail(IFDTD_ERR_UNSUPPORTED, "CUDA device index out of range");
  cudaDeviceProp prop;
  CUDA_TRY(cudaGetDeviceProperties(&prop, device));
  if (prop.major != 10) return fail(IFDTD_ERR_UNSUPPORTED, "this build targets sm_100a (B200)");
  DeviceGuard guard(device);
  ifdtd_plan* P = new ifdtd_plan();
  P->dtype = dtype_bytes;
  P->device = device;
  P->sm_count = prop.multiProcessorCount;
  const int rc = dtype_bytes == 4 ? build_plan<float>(P, mesh, grid, physics, tuning)
                                  : build_plan<double>(P, mesh, grid, physics, tuning);
  if (rc != IFDTD_OK) {
    delete P;
    return rc;
  }
  *out = P;
  return IFDTD_OK;
}

int32_t ifdtd_plan_destroy(ifdtd_plan* plan) {
  if (!plan) return IFDTD_OK;
  DeviceGuard guard(plan->device);
  cudaDeviceSynchronize();
  for (ifdtd_probe* p : plan->probes) p->plan = nullptr;
  delete plan;
  return IFDTD_OK;
}

int32_t ifdtd_plan_layout(const ifdtd_plan* plan, int32_t* node_pitch, int32_t* mid_pitch) {
  if (!plan || !node_pitch || !mid_pitch) return fail(IFDTD_ERR_ARGUMENT, "null argument");
  *node_pitch = plan->Pn;
  *mid_pitch = plan->Pm;
  return IFDTD_OK;
}

int32_t ifdtd_status_word(ifdtd_plan* plan, int32_t reset, int32_t* out) {
  if (!plan || !out) return fail(IFDTD_ERR_ARGUMENT, "null argument");
  DeviceGuard guard(plan->device);
  CUDA_TRY(cudaDeviceSynchronize());
  int value = 0;
  CUDA_TRY(cudaMemcpy(&value, plan->d_status, sizeof(int), cudaMemcpyDeviceToHost));
  if (reset) CUDA_TRY(cudaMemset(plan->d_status, 0, sizeof(int)));
  *out = value;
  return IFDTD_OK;
}

int32_t ifdtd_wait_selftest(ifdtd_plan* plan, double* waited_seconds, void* stream) {
  if (!plan || !waited_seconds) return fail(IFDTD_ERR_ARGUMENT, "null argument");
  DeviceGuard guard(plan->device);
  cudaStream_t st = (cudaStream_t)stream;
  unsigned long long* d_ns = nullptr;
  CUDA_TRY(cudaMalloc(&d_ns, sizeof(unsigned long long)));
  pipe::wait_selftest_kernel<<<1, 32, 0, st>>>(plan->d_status, d_ns);
  cudaError_t e = cudaGetLastError();
  unsigned long long ns = 0;
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e == cudaSuccess) e = cudaMemcpy(&ns, d_ns, sizeof(ns), cudaMemcpyDeviceToHost);
  cudaFree(d_ns);
  if (e != cudaSuccess) return fail(IFDTD_ERR_CUDA, std::string("wait self-test: ") + cudaGetErrorString(e));
  *waited_seconds = (double)ns * 1e-9;
  return IFDTD_OK;
}

int32_t ifdtd_plan_kernels(const ifdtd_plan* plan, int32_t* h_mode, int32_t* e_mode) {
  if (!plan || !h_mode || !e_mode) return fail(IFDTD_ERR_ARGUMENT, "null argument");
  *h_mode = plan->fused ? 3 : plan->h_mode;
  *e_mode = plan->fused ? (plan->fused_pipe ? 2 : 1) : plan->e_mode;
  return IFDTD_OK;
}

int32_t ifdtd_plan_bytes(const ifdtd_plan* plan, int64_t* bytes) {
  if (!plan || !bytes) return fail(IFDTD_ERR_ARGUMENT, "null argument");
  *bytes = (int64_t)plan->arena.bytes;
  return IFDTD_OK;
}

int32_t ifdtd_step(ifdtd_plan* plan, const ifdtd_state* state, const double* currents, int32_t n_steps, void* stream) {
  if (!plan) return fail(IFDTD_ERR_ARGUMENT, "null plan");
  if (n_steps < 0) return fail(IFDTD_ERR_ARGUMENT, "negative step count");
  DeviceGuard guard(plan->device);
  cudaStream_t st = (cudaStream_t)stream;
  return plan->dtype == 4 ? run_steps<float>(plan, state, currents, n_steps, nullptr, nullptr, st)
                          : run_steps<double>(plan, state, currents, n_steps, nullptr, nullptr, st);
}

int32_t ifdtd_update_magnetic(ifdtd_plan* plan, const ifdtd_state* state, void* stream) {
  if (!plan) return fail(IFDTD_ERR_ARGUMENT, "null plan");
  DeviceGuard guard(plan->device);
  cudaStream_t st = (cudaStream_t)stream;
  const int rc = plan->dtype == 4 ? bind_state<float>(plan, state, st) : bind_state<double>(plan, state, st);
  if (rc) return rc;
  CUDA_TRY(plan->dtype == 4 ? plasma_frames<float>(plan, state, 1, st) : plasma_frames<double>(plan, state, 1, st));
  CUDA_TRY(plan->dtype == 4 ? launch_kh<float>(plan, st) : launch_kh<double>(plan, st));
  CUDA_TRY(plan->dtype == 4 ? plasma_frames<float>(plan, state, 0, st) : plasma_frames<double>(plan, state, 0, st));
  CUDA_TRY(cudaGetLastError());
  return IFDTD_OK;
}

int32_t ifdtd_update_electric(ifdtd_plan* plan, const ifdtd_state* state, double current, void* stream) {
  if (!plan) return fail(IFDTD_ERR_ARGUMENT, "null plan");
  DeviceGuard guard(plan->device);
  cudaStream_t st = (cudaStream_t)stream;
  const int rc = plan->dtype == 4 ? bind_state<float>(plan, state, st) : bind_state<double>(plan, state, st);
  if (rc) return rc;
  // pageable source: staged by the runtime before the call returns
  CUDA_TRY(cudaMemcpyAsync(plan->d_cur, &current, sizeof(double), cudaMemcpyHostToDevice, st));
  CUDA_TRY(plan->dtype == 4 ? plasma_frames<float>(plan, state, 1, st) : plasma_frames<double>(plan, state, 1, st));
  CUDA_TRY(plan->dtype == 4 ? launch_ke<float>(plan, 0, st) : launch_ke<double>(plan, 0, st));
  CUDA_TRY(plan->dtype == 4 ? plasma_frames<float>(plan, state, 0, st) : plasma_frames<double>(plan, state, 0, st));
  CUDA_TRY(cudaGetLastError());
  return IFDTD_OK;
}

}  // extern "C"

namespace {

// Device time of each phase kernel: the state is turned into the plan's plasma
// frame once, the H and E phase kernels run 3 + reps times with a zero source
// current (CUDA events around every launch on the caller's stream), and the
// state is turned back.  Medians of the reps timed launches.
template <typename real>
int time_phases(ifdtd_plan* P, const ifdtd_state* s, int reps, float* h_ms, float* e_ms, cudaStream_t st) {
  int rc = bind_state<real>(P, s, st);
  if (rc) return rc;
  CUDA_TRY(cudaMemsetAsync(P->d_cur, 0, sizeof(double), st));
  CUDA_TRY(plasma_frames<real>(P, s, 1, st));
  for (int i = 0; i < 3; ++i) {
    CUDA_TRY(launch_kh<real>(P, st));
    CUDA_TRY(launch_ke<real>(P, 0, st));
  }
  std::vector<cudaEvent_t> ev(3 * (size_t)reps, nullptr);
  struct Events {
    std::vector<cudaEvent_t>& e;
    ~Events() {
      for (cudaEvent_t x : e)
        if (x) cudaEventDestroy(x);
    }
  } hold{ev};
  for (auto& x : ev) CUDA_TRY(cudaEventCreate(&x));
  for (int i = 0; i < reps; ++i) {
    CUDA_TRY(cudaEventRecord(ev[3 * i], st));
    CUDA_TRY(launch_kh<real>(P, st));
    CUDA_TRY(cudaEventRecord(ev[3 * i + 1], st));
    CUDA_TRY(launch_ke<real>(P, 0, st));
    CUDA_TRY(cudaEventRecord(ev[3 * i + 2], st));
  }
  CUDA_TRY(plasma_frames<real>(P, s, 0, st));
  CUDA_TRY(cudaEventSynchronize(ev.back()));
  std::vector<float> h(reps), e(reps);
  for (int i = 0; i < reps; ++i) {
    CUDA_TRY(cudaEventElapsedTime(&h[i], ev[3 * i], ev[3 * i + 1]));
    CUDA_TRY(cudaEventElapsedTime(&e[i], ev[3 * i + 1], ev[3 * i + 2]));
  }
  std::sort(h.begin(), h.end());
  std::sort(e.begin(), e.end());
  *h_ms = reps % 2 ? h[reps / 2] : 0.5f * (h[reps / 2 - 1] + h[reps / 2]);
  *e_ms = reps % 2 ? e[reps / 2] : 0.5f * (e[reps / 2 - 1] + e[reps / 2]);
  return IFDTD_OK;
}

}  // namespace

extern "C" {

int32_t ifdtd_time_phases(ifdtd_plan* plan, const ifdtd_state* state, int32_t reps, float* h_ms, float* e_ms,
                          void* stream) {
  if (!plan || !h_ms || !e_ms) return fail(IFDTD_ERR_ARGUMENT, "null argument");
  if (reps < 1) return fail(IFDTD_ERR_ARGUMENT, "reps must be positive");
  DeviceGuard guard(plan->device);
  cudaStream_t st = (cudaStream_t)stream;
  return plan->dtype == 4 ? time_phases<float>(plan, state, reps, h_ms, e_ms, st)
                          : time_phases<double>(plan, state, reps, h_ms, e_ms, st);
}

int32_t ifdtd_probe_create(ifdtd_plan* plan, int32_t field_kind, int32_t rows, int32_t width, const int64_t* index,
                           const int64_t* layer, const double* weight, ifdtd_probe** out) {
  if (!plan || !out || !index || !layer || !weight) return fail(IFDTD_ERR_ARGUMENT, "null argument");
  if (field_kind < 0 || field_kind > 3 || rows <= 0 || width <= 0) return fail(IFDTD_ERR_ARGUMENT, "bad probe shape");
  const int64_t n_ent = field_kind == 0 ? plan->nV : field_kind == 2 ? plan->nF : plan->nE;
  const int64_t n_lay = (field_kind == 0 || field_kind == 3) ? plan->L + 1 : plan->L;
  const size_t n = (size_t)rows * width;
  std::vector<int> idx(n), lay(n);
  std::vector<double> w(weight, weight + n);
  for (size_t i = 0; i < n; ++i) {
    if (index[i] < 0 || index[i] >= n_ent || layer[i] < 0 || layer[i] >= n_lay)
      return fail(IFDTD_ERR_ARGUMENT, "probe index out of range");
    idx[i] = (int)index[i];
    lay[i] = (int)layer[i];
  }
  DeviceGuard guard(plan->device);
  ifdtd_probe* p = new ifdtd_probe();
  p->plan = plan;
  p->kind = field_kind;
  p->rows = rows;
  p->width = width;
  const int* di = nullptr;
  const int* dl = nullptr;
  const double* dw = nullptr;
  void* stg = nullptr;
  if (p->arena.upload(idx, &di) != cudaSuccess || p->arena.upload(lay, &dl) != cudaSuccess ||
      p->arena.upload(w, &dw) != cudaSuccess ||
      p->arena.alloc((size_t)std::max(plan->chunk, 1) * rows * sizeof(double), &stg) != cudaSuccess) {
    delete p;
    return fail(IFDTD_ERR_CUDA, "probe upload failed");
  }
  p->index = (int*)di;
  p->layer = (int*)dl;
  p->weight = (double*)dw;
  p->staging = (double*)stg;
  plan->probes.push_back(p);
  *out = p;
  return IFDTD_OK;
}

int32_t ifdtd_probe_destroy(ifdtd_probe* probe) {
  // the probe's buffers are released with it; graphs that sample it are dropped
  if (!probe) return IFDTD_OK;
  if (probe->plan) {
    DeviceGuard guard(probe->plan->device);
    cudaDeviceSynchronize();
    auto& v = probe->plan->probes;
    v.erase(std::remove(v.begin(), v.end(), probe), v.end());
    auto& g = probe->plan->graphs;
    for (auto it = g.begin(); it != g.end();) {
      if (it->probe == probe) {
        cudaGraphExecDestroy(it->exec);
        it = g.erase(it);
      } else {
        ++it;
      }
    }
  }
  delete probe;
  return IFDTD_OK;
}

int32_t ifdtd_sample(ifdtd_plan* plan, const ifdtd_state* state, const ifdtd_probe* probe, double* out_row,
                     void* stream) {
  if (!plan || !probe || !out_row || probe->plan != plan) return fail(IFDTD_ERR_ARGUMENT, "bad sample arguments");
  DeviceGuard guard(plan->device);
  cudaStream_t st = (cudaStream_t)stream;
  const int rc = plan->dtype == 4 ? bind_state<float>(plan, state, st) : bind_state<double>(plan, state, st);
  if (rc) return rc;
  const void* field = probe->kind == 0 ? state->er : probe->kind == 1 ? state->et : probe->kind == 2 ? state->hr : state->ht;
  const int pitch = (probe->kind == 0 || probe->kind == 3) ? plan->Pn : plan->Pm;
  const int blocks = (probe->rows * 32 + 255) / 256;
  if (plan->dtype == 4)
    sample_kernel<float><<<blocks, 256, 0, st>>>((const float*)field, pitch, probe->rows, probe->width, probe->index,
                                                 probe->layer, probe->weight, out_row);
  else
    sample_kernel<double><<<blocks, 256, 0, st>>>((const double*)field, pitch, probe->rows, probe->width,
                                                  probe->index, probe->layer, probe->weight, out_row);
  CUDA_TRY(cudaGetLastError());
  return IFDTD_OK;
}

int32_t ifdtd_step_sampled(ifdtd_plan* plan, const ifdtd_state* state, const double* currents, int32_t n_steps,
                           const ifdtd_probe* probe, double* out_rows, void* stream) {
  if (!plan || !probe || !out_rows || probe->plan != plan) return fail(IFDTD_ERR_ARGUMENT, "bad sampled-step arguments");
  if (n_steps < 0) return fail(IFDTD_ERR_ARGUMENT, "negative step count");
  DeviceGuard guard(plan->device);
  cudaStream_t st = (cudaStream_t)stream;
  return plan->dtype == 4 ? run_steps<float>(plan, state, currents, n_steps, probe, out_rows, st)
                          : run_steps<double>(plan, state, currents, n_steps, probe, out_rows, st);
}

int32_t ifdtd_first_use_numbering(const int64_t* lo, const int64_t* hi, int64_t n, int64_t n_vertices, int64_t* rank,
                                  int64_t* first, int64_t* n_distinct) {
  if (!n_distinct || n < 0 || n_vertices <= 0 || n_vertices >= ((int64_t)1 << 31) ||
      (n > 0 && (!lo || !hi || !rank || !first)))
    return fail(IFDTD_ERR_ARGUMENT, "bad first-use numbering arguments");
  // open addressing on key = lo * n_vertices + hi, table at least twice the pairs
  int shift = 64 - 4;
  size_t cap = 16;
  while (cap < 2 * (size_t)n) {
    cap <<= 1;
    --shift;
  }
  std::vector<int64_t> keys(cap, -1), ranks(cap, 0);
  int64_t count = 0;
  for (int64_t i = 0; i < n; ++i) {
    if (lo[i] < 0 || hi[i] < 0 || lo[i] >= n_vertices || hi[i] >= n_vertices)
      return fail(IFDTD_ERR_ARGUMENT, "vertex index out of range in first-use numbering");
    const int64_t key = lo[i] * n_vertices + hi[i];
    size_t h = (size_t)(((uint64_t)key * 0x9E3779B97F4A7C15ull) >> shift);
    while (keys[h] != -1 && keys[h] != key) h = (h + 1) & (cap - 1);
    if (keys[h] == -1) {
      keys[h] = key;
      ranks[h] = count;
      first[count++] = i;
    }
    rank[i] = ranks[h];
  }
  *n_distinct = count;
  return IFDTD_OK;
}

int32_t ifdtd_stable_group(const int64_t* keys, int64_t n, int64_t n_keys, int64_t* order, int64_t* counts) {
  if (n < 0 || n_keys <= 0 || !counts || (n > 0 && (!keys || !order)))
    return fail(IFDTD_ERR_ARGUMENT, "bad stable grouping arguments");
  std::fill(counts, counts + n_keys, (int64_t)0);
  for (int64_t i = 0; i < n; ++i) {
    if (keys[i] < 0 || keys[i] >= n_keys) return fail(IFDTD_ERR_ARGUMENT, "key out of range in stable grouping");
    ++counts[keys[i]];
  }
  // counting sort: each group's first free position, filled in position order
  std::vector<int64_t> next((size_t)n_keys);
  int64_t at = 0;
  for (int64_t k = 0; k < n_keys; ++k) {
    next[(size_t)k] = at;
    at += counts[k];
  }
  for (int64_t i = 0; i < n; ++i) order[next[(size_t)keys[i]]++] = i;
  return IFDTD_OK;
}

int32_t ifdtd_batch_create(ifdtd_plan* const* plans, int32_t n_members, int32_t chunk, ifdtd_batch** out) {
  if (!plans || !out || n_members <= 0 || chunk < 1) return fail(IFDTD_ERR_ARGUMENT, "bad batch arguments");
  *out = nullptr;
  for (int i = 0; i < n_members; ++i) {
    if (!plans[i]) return fail(IFDTD_ERR_ARGUMENT, "null member plan");
    if (plans[i]->device != plans[0]->device || plans[i]->dtype != plans[0]->dtype)
      return fail(IFDTD_ERR_ARGUMENT, "batch members must share one device and one precision");
    for (int j = 0; j < i; ++j)
      if (plans[j] == plans[i]) return fail(IFDTD_ERR_ARGUMENT, "a plan appears twice in the batch");
  }
  DeviceGuard guard(plans[0]->device);
  ifdtd_batch* B = new ifdtd_batch();
  B->device = plans[0]->device;
  B->dtype = plans[0]->dtype;
  B->n = n_members;
  B->plans.assign(plans, plans + n_members);
  B->chunk = chunk;
  bool fused = false;
  for (int i = 0; i < n_members; ++i) {
    if (plans[i]->h_mode != 2 || plans[i]->e_mode != 2) B->chunk = std::min(B->chunk, std::max(plans[i]->chunk, 1));
    fused |= plans[i]->fused;
  }
  if (fused && B->chunk % 2) {
    delete B;
    return fail(IFDTD_ERR_ARGUMENT, "a batch with fused-step members needs an even chunk");
  }
  const int rc = B->dtype == 4 ? batch_build<float>(B) : batch_build<double>(B);
  if (rc) {
    delete B;
    return rc;
  }
  *out = B;
  return IFDTD_OK;
}

int32_t ifdtd_batch_destroy(ifdtd_batch* batch) {
  if (!batch) return IFDTD_OK;
  DeviceGuard guard(batch->device);
  cudaDeviceSynchronize();
  delete batch;
  return IFDTD_OK;
}

int32_t ifdtd_batch_step(ifdtd_batch* batch, const ifdtd_state* states, const double* currents, int32_t n_steps,
                         ifdtd_probe* const* probes, double* const* out_rows, void* stream) {
  if (!batch || !states) return fail(IFDTD_ERR_ARGUMENT, "null argument");
  if (n_steps < 0) return fail(IFDTD_ERR_ARGUMENT, "negative step count");
  DeviceGuard guard(batch->device);
  cudaStream_t st = (cudaStream_t)stream;
  return batch->dtype == 4 ? run_batch<float>(batch, states, currents, n_steps, probes, out_rows, st)
                           : run_batch<double>(batch, states, currents, n_steps, probes, out_rows, st);
}

int32_t ifdtd_batch_info(const ifdtd_batch* batch, int32_t* groups, int32_t* solo, int32_t* kh_grid,
                         int32_t* ke_grid) {
  if (!batch || !groups || !solo || !kh_grid || !ke_grid) return fail(IFDTD_ERR_ARGUMENT, "null argument");
  *groups = (int32_t)batch->groups.size();
  *solo = (int32_t)batch->solo.size();
  *kh_grid = batch->groups.empty() ? 0 : batch->groups[0].kh_grid;
  *ke_grid = batch->groups.empty() ? 0 : batch->groups[0].ke_grid;
  return IFDTD_OK;
}

int32_t ifdtd_max_abs(ifdtd_plan* plan, const ifdtd_state* state, double* out4, void* stream) {
  if (!plan || !state || !out4) return fail(IFDTD_ERR_ARGUMENT, "null argument");
  DeviceGuard guard(plan->device);
  cudaStream_t st = (cudaStream_t)stream;
  CUDA_TRY(cudaMemsetAsync(out4, 0, 4 * sizeof(double), st));
  const size_t n0 = (size_t)plan->nV * plan->Pn, n1 = (size_t)plan->nE * plan->Pm;
  const size_t n2 = (size_t)plan->nF * plan->Pm, n3 = (size_t)plan->nE * plan->Pn;
  dim3 grid(grid_for(std::max(std::max(n0, n1), std::max(n2, n3))), 4);
  if (plan->dtype == 4)
    max_abs_kernel<float><<<grid, 256, 0, st>>>((const float*)state->er, n0, (const float*)state->et, n1,
                                                (const float*)state->hr, n2, (const float*)state->ht, n3,
                                                (unsigned long long*)out4);
  else
    max_abs_kernel<double><<<grid, 256, 0, st>>>((const double*)state->er, n0, (const double*)state->et, n1,
                                                 (const double*)state->hr, n2, (const double*)state->ht, n3,
                                                 (unsigned long long*)out4);
  CUDA_TRY(cudaGetLastError());
  return IFDTD_OK;
}

#define PRIM_PROLOGUE                                                        \
  if (!plan || !in || !out || cols <= 0) return fail(IFDTD_ERR_ARGUMENT, "bad primitive arguments"); \
  DeviceGuard guard(plan->device);                                           \
  cudaStream_t st = (cudaStream_t)stream;

int32_t ifdtd_edge_difference(ifdtd_plan* plan, const void* in, int32_t cols, void* out, void* stream) {
  PRIM_PROLOGUE
  const int g = grid_for((size_t)plan->nE * cols);
  if (plan->dtype == 4)
    pair_difference_kernel<float><<<g, 256, 0, st>>>((const float*)in, cols, plan->nE, plan->edge_th, false, (float*)out);
  else
    pair_difference_kernel<double><<<g, 256, 0, st>>>((const double*)in, cols, plan->nE, plan->edge_th, false,
                                                      (double*)out);
  CUDA_TRY(cudaGetLastError());
  return IFDTD_OK;
}

int32_t ifdtd_dual_edge_difference(ifdtd_plan* plan, const void* in, int32_t cols, void* out, void* stream) {
  PRIM_PROLOGUE
  const int g = grid_for((size_t)plan->nE * cols);
  if (plan->dtype == 4)
    pair_difference_kernel<float><<<g, 256, 0, st>>>((const float*)in, cols, plan->nE, plan->edge_lr, true, (float*)out);
  else
    pair_difference_kernel<double><<<g, 256, 0, st>>>((const double*)in, cols, plan->nE, plan->edge_lr, true,
                                                      (double*)out);
  CUDA_TRY(cudaGetLastError());
  return IFDTD_OK;
}

int32_t ifdtd_face_circulation(ifdtd_plan* plan, const void* in, int32_t cols, void* out, void* stream) {
  PRIM_PROLOGUE
  const int g = grid_for((size_t)plan->nF * cols);
  if (plan->dtype == 4)
    face_circulation_kernel<float><<<g, 256, 0, st>>>((const float*)in, cols, plan->nF, plan->face_e, plan->face_sign,
                                                      (float*)out);
  else
    face_circulation_kernel<double><<<g, 256, 0, st>>>((const double*)in, cols, plan->nF, plan->face_e,
                                                       plan->face_sign, (double*)out);
  CUDA_TRY(cudaGetLastError());
  return IFDTD_OK;
}

int32_t ifdtd_dual_cell_circulation(ifdtd_plan* plan, const void* in, int32_t cols, void* out, void* stream) {
  PRIM_PROLOGUE
  const int g = grid_for((size_t)plan->nV * cols);
  if (plan->dtype == 4)
    dual_cell_circulation_kernel<float><<<g, 256, 0, st>>>((const float*)in, cols, plan->nV, plan->v_off, plan->v_edge,
                                                           plan->v_sign, (float*)out);
  else
    dual_cell_circulation_kernel<double><<<g, 256, 0, st>>>((const double*)in, cols, plan->nV, plan->v_off,
                                                            plan->v_edge, plan->v_sign, (double*)out);
  CUDA_TRY(cudaGetLastError());
  return IFDTD_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free stepping (no counterpart in the reference).
//
// Some callers may not allocate device memory while they run: a process that
// hands all free device memory to its own pool at start-up (cudaMalloc would
// then fail), or a latency-bound loop that cannot afford the device-wide
// synchronisation that cudaMalloc and cudaFree may perform.  They use
// ifdtd_step_static_scratch.  A multi-species plasma step needs one scratch
// buffer, the summed species current (F x 3 x mid_pitch reals) that the H
// kernel writes and the E kernel reads; the plan allocates it with cudaMalloc.
// Here it lives in a file-scope device array of kStaticScratchBytes instead,
// together with a device copy of the launch record that points the kernels
// at it.  Every GPU that loads this library holds both arrays until the
// process exits.  In host code the arrays' names are host-side stand-ins, so
// their device addresses are looked up once per device (with that device
// current) by cudaGetSymbolAddress and passed to the kernels.
// ---------------------------------------------------------------------------
namespace {

constexpr size_t kStaticScratchBytes = (size_t)16 << 20;  // summed plasma current
constexpr int kStaticMaxDevices = 64;
static_assert(sizeof(Rec<double>) >= sizeof(Rec<float>), "record size");

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];
static __device__ __align__(256) unsigned char g_static_record[sizeof(Rec<double>)];
static __device__ __align__(256) double g_static_zero_current[1];

// Per device: the arrays' device addresses and a host copy of the record last
// uploaded to g_static_record (uploaded = false until the first upload).  The
// mutex makes the first lookup and the record comparison safe when several
// host threads call on the same device.
struct StaticDevice {
  std::mutex lock;
  bool ready = false;
  void* scratch = nullptr;
  void* record = nullptr;
  void* zero_current = nullptr;
  bool uploaded = false;
  unsigned char last_record[sizeof(Rec<double>)];
};
StaticDevice g_static_devices[kStaticMaxDevices];

// Device addresses of the static arrays on `device` (which must be current);
// looked up on the first call for that device.  The caller holds a.lock.
int static_addresses(StaticDevice& a) {
  if (a.ready) return IFDTD_OK;
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
  if (e != cudaSuccess) return fail(IFDTD_ERR_CUDA, std::string("static scratch address: ") + cudaGetErrorString(e));
  a.scratch = p;
  e = cudaGetSymbolAddress(&p, g_static_record);
  if (e != cudaSuccess) return fail(IFDTD_ERR_CUDA, std::string("static record address: ") + cudaGetErrorString(e));
  a.record = p;
  e = cudaGetSymbolAddress(&p, g_static_zero_current);
  if (e != cudaSuccess) return fail(IFDTD_ERR_CUDA, std::string("static current address: ") + cudaGetErrorString(e));
  a.zero_current = p;
  a.ready = true;
  return IFDTD_OK;
}

template <typename real>
int step_static(ifdtd_plan* P, const ifdtd_state* st, const double* currents, int n, cudaStream_t stream) {
  const size_t need = P->S > 1 ? (size_t)P->nF * 3 * P->Pm * sizeof(real) : 0;
  if (need > kStaticScratchBytes)
    return fail(IFDTD_ERR_UNSUPPORTED, "ifdtd_step_static_scratch: the summed plasma current needs " +
                                           std::to_string(need) + " bytes, above the " +
                                           std::to_string(kStaticScratchBytes) + "-byte static scratch");
  if (P->device < 0 || P->device >= kStaticMaxDevices) return fail(IFDTD_ERR_UNSUPPORTED, "device ordinal too large");
  int rc = bind_state<real>(P, st, stream);
  if (rc) return rc;
  if (n <= 0) return IFDTD_OK;
  StaticDevice& A = g_static_devices[P->device];
  std::lock_guard<std::mutex> hold(A.lock);
  rc = static_addresses(A);
  if (rc) return rc;
  // the plan's record with the summed current and the source row pointed at
  // the static arrays; the bytes not covered by Rec<real> stay zero
  unsigned char bytes[sizeof(Rec<double>)] = {};
  Rec<real> rec;
  std::memcpy(&rec, P->h_rec.data(), sizeof(rec));
  rec.Jtot = P->S > 1 ? static_cast<real*>(A.scratch) : nullptr;
  rec.cur = currents ? currents : static_cast<const double*>(A.zero_current);
  std::memcpy(bytes, &rec, sizeof(rec));
  // the summed current is fully rewritten each step; clearing it keeps a call
  // independent of what the previous call left behind
  if (need) CUDA_TRY(cudaMemsetAsync(A.scratch, 0, need, stream));
  if (!currents) CUDA_TRY(cudaMemsetAsync(A.zero_current, 0, sizeof(double), stream));
  if (!A.uploaded || std::memcmp(A.last_record, bytes, sizeof(bytes)) != 0) {
    // pageable source: copied to staging before the call returns
    CUDA_TRY(cudaMemcpyAsync(A.record, bytes, sizeof(bytes), cudaMemcpyHostToDevice, stream));
    std::memcpy(A.last_record, bytes, sizeof(bytes));
    A.uploaded = true;
  }
  const Rec<real>* drec = static_cast<const Rec<real>*>(A.record);
  CUDA_TRY(plasma_frames<real>(P, st, 1, stream));
  for (int i = 0; i < n; ++i) {
    cudaError_t e = P->plasma ? launch_kh_t<real, true>(P, drec, stream) : launch_kh_t<real, false>(P, drec, stream);
    if (e == cudaSuccess) {
      const int istep = currents ? i : 0;
      if (P->maxdeg == 6)
        e = P->plasma ? launch_ke_t<real, true, 6>(P, drec, istep, stream)
                      : launch_ke_t<real, false, 6>(P, drec, istep, stream);
      else
        e = P->plasma ? launch_ke_t<real, true, 12>(P, drec, istep, stream)
                      : launch_ke_t<real, false, 12>(P, drec, istep, stream);
    }
    if (e != cudaSuccess) return fail(IFDTD_ERR_CUDA, std::string("static-scratch step launch: ") + cudaGetErrorString(e));
  }
  CUDA_TRY(plasma_frames<real>(P, st, 0, stream));
  return IFDTD_OK;
}

}  // namespace

extern "C" int32_t ifdtd_step_static_scratch(ifdtd_plan* plan, const ifdtd_state* state, const double* currents,
                                             int32_t n_steps, void* stream) {
  if (!plan) return fail(IFDTD_ERR_ARGUMENT, "null plan");
  if (n_steps < 0) return fail(IFDTD_ERR_ARGUMENT, "negative step count");
  DeviceGuard guard(plan->device);
  cudaStream_t st = (cudaStream_t)stream;
  return plan->dtype == 4 ? step_static<float>(plan, state, currents, n_steps, st)
                          : step_static<double>(plan, state, currents, n_steps, st);
}
