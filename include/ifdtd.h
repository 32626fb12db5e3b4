/*
 * ifdtd.h - C ABI of the B200 geodesic FDTD time-step engine.
 *
 * The reference (ruddyscent/ionosphere-fdtd v0.2.0) is pure Python: its
 * time-step path is GeodesicFDTD.step (src/ionosphere_fdtd/solver.py:789-816)
 * running on the ArrayBackend seam (src/ionosphere_fdtd/backends/base.py:19-89,
 * selected by create_backend in backends/__init__.py:12-33).  There is no FFI
 * in the reference; each entry point below names the reference interface it
 * replaces.  All pointers are plain host or device pointers, all sizes are
 * plain integers, and no torch type appears.  Every function returns an
 * ifdtd_status; ifdtd_last_error() gives the message of the last failure on
 * the calling thread.
 *
 * Layout contract: every field is a row-major (entity, radial) array with the
 * radial index contiguous, as the reference's er (V, L+1), et (E, L),
 * hr (F, L), ht (E, L+1) arrays (solver.py:315-322), but with a row pitch
 * chosen by the plan (ifdtd_plan_layout): node arrays er/ht use node_pitch
 * >= L+1, midpoint arrays et/hr use mid_pitch >= L, both multiples of 16
 * bytes, so that every radial run is one aligned 16-byte vector access.  The
 * padding elements of a row must be zero on entry and stay zero.  Plasma
 * current densities, (F, L, 3) per species in the reference (plasma.py:411),
 * are stored component-major as (F, 3, mid_pitch).  Surface-impedance memory
 * is (E, T) (surface_impedance.py:203).  Base pointers are 16-byte aligned.
 * Element type is float (dtype 4) or double (dtype 8) for a whole plan.
 */
#ifndef IFDTD_H
#define IFDTD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define IFDTD_MAX_SPECIES 4
#define IFDTD_MAX_SOURCES 16

typedef enum ifdtd_status {
  IFDTD_OK = 0,
  IFDTD_ERR_ARGUMENT = 1,   /* invalid argument (maps to ValueError) */
  IFDTD_ERR_CUDA = 2,       /* CUDA runtime failure (maps to RuntimeError) */
  IFDTD_ERR_NONFINITE = 3,  /* a field holds NaN/Inf (diagnostics) */
  IFDTD_ERR_UNSUPPORTED = 4 /* feature or device not supported (BackendUnavailableError) */
} ifdtd_status;

typedef struct ifdtd_plan ifdtd_plan;
typedef struct ifdtd_probe ifdtd_probe;
typedef struct ifdtd_batch ifdtd_batch;

/* Mesh tables as GeodesicMesh holds them (src/ionosphere_fdtd/mesh.py:21-41). */
typedef struct ifdtd_mesh_desc {
  int32_t n_vertices, n_edges, n_faces;
  const int64_t* edges;            /* (E,2) tail, head            mesh.py:27  */
  const int64_t* faces;            /* (F,3) outward-oriented      mesh.py:26  */
  const int64_t* face_edges;       /* (F,3)                       mesh.py:28  */
  const int64_t* face_edge_signs;  /* (F,3) +1 / -1               mesh.py:29  */
  const int64_t* edge_left_faces;  /* (E)                         mesh.py:30  */
  const int64_t* edge_right_faces; /* (E)                         mesh.py:31  */
  const double* primal_edge_angles;     /* (E) theta              mesh.py:33 */
  const double* dual_edge_angles;       /* (E) phi                mesh.py:34 */
  const double* face_solid_angles;      /* (F) A_f                mesh.py:35 */
  const double* dual_cell_solid_angles; /* (V) A*_v               mesh.py:36 */
} ifdtd_mesh_desc;

/* Radial grid and integration controls (solver.py:260-283, 296-300). */
typedef struct ifdtd_grid_desc {
  int32_t radial_cells;   /* L; nodes 0..L, midpoints 0..L-1 */
  int32_t full_spherical; /* geometry_mode == "full-spherical" */
  const double* radii_m;  /* (L+1) node radii */
  double time_step_s;
} ifdtd_grid_desc;

/* Physics coefficients built by the host exactly as the reference builds them:
 * loss coefficients (solver.py:706-761), source supports (solver.py:936-987,
 * sources.py:220-235, 290-335), surface-impedance ADE (surface_impedance.py:
 * 176-203), plasma ADE and coupler tables (plasma.py:374-411, 458-487). */
typedef struct ifdtd_physics_desc {
  /* loss coefficients; rows = 1 (altitude-only profile) or V / E */
  int32_t coef_rows_er, coef_rows_et;
  const double *ca_er, *cb_er; /* (rows, L+1) */
  const double *ca_et, *cb_et; /* (rows, L)   */
  /* vertical source: er[v,k] -= coef * I(step); tangential: et[e,j] -= coef * I */
  int32_t n_src_er;
  const int64_t *src_er_vertex, *src_er_layer;
  const double* src_er_coef;
  int32_t n_src_et;
  const int64_t *src_et_edge, *src_et_layer;
  const double* src_et_coef;
  /* lower surface-impedance ADE (terms = 0 disables) */
  int32_t si_terms;
  const double* si_scale;    /* (E) sqrt(mu / sigma_e) */
  const double* si_decay;    /* (T) (1-a)/(1+a) */
  const double* si_drive;    /* (T) a/(1+a)     */
  const double* si_history;  /* (T) w/(1+a)     */
  double si_metric;          /* m_0 / r_0 (full-spherical) or 1 */
  /* cold-plasma ADE (species = 0 disables) */
  int32_t plasma_species;
  int32_t plasma_rows;       /* 1 (altitude-only) or F */
  int32_t plasma_magnetized; /* 0: b = 0 everywhere */
  const double* plasma_coef; /* (S, 6, rows, L): decay, cos, sin, d_par, d_re, d_im */
  const double* plasma_bdir; /* (rows, L, 3) unit B (magnetized only) */
  const double* plasma_reconstruction; /* (F,3,3) pinv(tangents).T per face */
  const double* face_centers;          /* (F,3) */
  const double* plasma_tangent_left;   /* (E,3) */
  const double* plasma_tangent_right;  /* (E,3) */
  int32_t vertex_face_width;           /* W */
  const int64_t* vertex_faces;         /* (V,W) padded with weight 0 */
  const double* vertex_face_weights;   /* (V,W) */
} ifdtd_physics_desc;

/* Tuning of the launch geometry (0 = defaults). */
typedef struct ifdtd_tuning {
  int32_t faces_per_patch;   /* faces owned by one H-phase patch (0: fit the pipeline stage to shared memory) */
  int32_t threads;           /* threads per direct CTA, or compute threads per pipelined CTA (0: automatic) */
  int32_t graph_chunk;       /* steps captured per CUDA graph (default 32; 0 disables) */
  int32_t e_faces_per_patch; /* faces whose vertices/edges one E-phase patch owns (0: fit the stage to shared memory) */
  int32_t staging;           /* 0 auto, 1 direct global gathers, 2 pipeline (TMA bulk copies), 3 pipeline (cp.async) */
  int32_t producer_warps;    /* copy-issuing warps per pipelined CTA (default 2, at most 4) */
  int32_t lane_layout;       /* pipelined consumers: 0 auto (packed), 1 rows packed back to back across lanes,
                                2 every row starting on an 8-lane boundary (no shared-memory bank conflicts
                                between rows; rows stay packed when a rounded-up row exceeds the threads) */
  int32_t e_threads;         /* compute threads of a pipelined E-phase CTA (0: as threads); with the producer
                                warps above 384 the E phase runs wide CTAs at 96 registers (at most 640
                                threads, TMA bulk copies only) */
  int32_t e_stages;          /* E-phase ring stages the balanced patches are sized for (0: 2, else 2 to 4) */
  int32_t e_producer_warps;  /* copy-issuing warps of a pipelined E-phase CTA (0: 4 when threads and e_threads
                                are automatic, else as producer_warps; or 1 to 4) */
  int32_t e_copy_gap;        /* E-phase copies: gaps of up to this many rows (0 to 8) between staged rows of one
                                array are always copied over, giving fewer and longer bulk copies */
  int32_t fused_step;        /* 1: one launch per leapfrog step, each E-phase patch recomputing the new H it
                                reads on its halo (plans without plasma or surface impedance; the plan holds a
                                second copy of the four field arrays and alternates between the copies, copying
                                back after an odd number of steps; graph_chunk must be even; in a batch (even
                                chunk) it runs the batched ring kernel).  staging 0 / 2 / 3: patches staged
                                through the pipelined ring
                                (TMA bulk copies / cp.async), the new H overwriting the old in the stage;
                                staging 1: direct gathers with the halo's new H in shared memory.
                                e_faces_per_patch sets the patch (0: the largest of 64 ... 8 faces whose stage
                                fits twice, direct: of 128 ... 16 faces whose rows fit 110 KiB); 0: two launches */
  int32_t plasma_frame;      /* frame the plasma current is held in while the step kernels run: 0 auto (face
                                frames for an unmagnetised plasma, else Cartesian), 1 Cartesian, 2 face frames
                                (unmagnetised plasma only).  In face frames component 0 lies along the face
                                centre and 1, 2 in the face's tangent plane, so the E phase reads one current
                                row per face at a vertex and two per face at an edge.  Every call that runs a
                                plasma phase turns the caller's Cartesian currents into face frames first and
                                back afterwards (two passes over the currents per call), so the state between
                                calls is the reference's (a call that fails part-way may leave the currents in
                                face frames, like its other results invalid); the two frames round differently
                                (float32: within a few ulp of the current per call) */
} ifdtd_tuning;

/* Mutable state of one simulation: device pointers owned by the caller. */
typedef struct ifdtd_state {
  void *er, *et, *hr, *ht;
  void* si_memory;                          /* (E,T) or NULL */
  void* plasma_current[IFDTD_MAX_SPECIES];  /* (F,3,mid_pitch) each */
} ifdtd_state;

int32_t ifdtd_version(void);
int32_t ifdtd_last_error(char* buffer, size_t size);
int32_t ifdtd_device_count(int32_t* count);

/* Build a plan for one simulation: uploads derived device tables
 * (replaces GeodesicFDTD.__init__'s backend setup, solver.py:238-375). */
int32_t ifdtd_plan_create(const ifdtd_mesh_desc* mesh, const ifdtd_grid_desc* grid,
                          const ifdtd_physics_desc* physics, const ifdtd_tuning* tuning,
                          int32_t dtype_bytes, int32_t device, ifdtd_plan** out);
int32_t ifdtd_plan_destroy(ifdtd_plan* plan);
/* Row pitches (in elements) the plan expects for node and midpoint arrays. */
int32_t ifdtd_plan_layout(const ifdtd_plan* plan, int32_t* node_pitch, int32_t* mid_pitch);
/* Device status word: bit 0 set when a wait of the pipelined kernels ran out
 * its time bound (the step's results are then invalid).  Reading it
 * synchronises the plan's device; reset != 0 clears it. */
int32_t ifdtd_status_word(ifdtd_plan* plan, int32_t reset, int32_t* out);
/* Test hook for failure detection (no counterpart in the reference): runs one
 * bounded wait of the pipelined kernels on an mbarrier that nothing completes.
 * The wait gives up after its time bound (0.5 s), sets bit 0 of the plan's
 * status word and returns; waited_seconds receives the time it waited.
 * Synchronises the stream. */
int32_t ifdtd_wait_selftest(ifdtd_plan* plan, double* waited_seconds, void* stream);
/* Which step kernels the plan launches: 1 direct gathers, 2 shared-memory
 * pipeline (H phase, E phase); h_mode 3: the fused one-launch step, whose
 * kernel family e_mode gives. */
int32_t ifdtd_plan_kernels(const ifdtd_plan* plan, int32_t* h_mode, int32_t* e_mode);
/* Bytes of device memory held by the plan (tables, staging, scratch). */
int32_t ifdtd_plan_bytes(const ifdtd_plan* plan, int64_t* bytes);

/* Advance n_steps leapfrog steps in place; currents (device, float64,
 * n_steps) are the source waveform I((n+1/2)dt) per step.  Replaces
 * GeodesicFDTD.step / _advance_fields / _advance_field_chunk
 * (solver.py:789-816, 867-875) and the backend compile_step hook
 * (backends/base.py:27-34, torch_backend.py:91-96). */
int32_t ifdtd_step(ifdtd_plan* plan, const ifdtd_state* state, const double* currents,
                   int32_t n_steps, void* stream);

/* Same as ifdtd_step, but allocates no device memory in any call.  It has no
 * counterpart in the reference.  It is for callers that may not call
 * cudaMalloc while they run: a process that hands all free device memory to
 * its own pool at start-up (cudaMalloc would fail there), or a latency-bound
 * loop that cannot afford the device-wide synchronisation cudaMalloc and
 * cudaFree may perform.  Do not call it from a CUDA stream callback (host
 * functions enqueued on a stream may make no CUDA calls).  The scratch that
 * a step with more than one plasma species needs (the summed current,
 * F x 3 x mid_pitch reals) lives in a 16 MiB static device array that every
 * GPU loading this library holds until exit; larger meshes are rejected with
 * IFDTD_ERR_UNSUPPORTED before any device work.  currents may be NULL (zero
 * source).  The first call on a device looks up the static arrays' device
 * addresses, so make it before any stream capture.  A call whose launch
 * record differs from the one last uploaded on that device (another plan,
 * other state or currents pointers) copies the record from host memory.  All
 * calls share the static arrays, which keep the last call's contents: calls
 * that overlap on the GPU (other streams, other plans) race and must be
 * serialised by the caller.  The first lookup and the record comparison are
 * guarded per device, so calls from several host threads leave that host
 * state intact; the race on the GPU above still applies to them. */
int32_t ifdtd_step_static_scratch(ifdtd_plan* plan, const ifdtd_state* state, const double* currents,
                                  int32_t n_steps, void* stream);

/* The two half steps of one leapfrog step, for callers that drive them
 * separately: the magnetic update (solver.py:877-921) and the electric update
 * with source current I (solver.py:923-989).  ifdtd_step is the pair. */
int32_t ifdtd_update_magnetic(ifdtd_plan* plan, const ifdtd_state* state, void* stream);
int32_t ifdtd_update_electric(ifdtd_plan* plan, const ifdtd_state* state, double current, void* stream);

/* Measurement helper (no counterpart in the reference): device time of the
 * H and E phase kernels, each launch bracketed by CUDA events on the stream;
 * the medians of reps timed launches (after 3 untimed pairs) go to h_ms and
 * e_ms.  Advances the state by 3 + reps leapfrog steps with a zero source
 * current; the plasma current is turned into the plan's frame once around all
 * of them, so the times are the phase kernels' alone.  Synchronises on the
 * last event. */
int32_t ifdtd_time_phases(ifdtd_plan* plan, const ifdtd_state* state, int32_t reps, float* h_ms, float* e_ms,
                          void* stream);

/* Weighted observation probe: out[r] = sum_k w[r,k] * field[index[r,k], layer[r,k]]
 * accumulated in float64.  field_kind: 0 er, 1 et, 2 hr, 3 ht.  Replaces the
 * sampling closures of record_er_observations / record_h_observations
 * (solver.py:1122-1124, 1212-1220). */
int32_t ifdtd_probe_create(ifdtd_plan* plan, int32_t field_kind, int32_t rows, int32_t width,
                           const int64_t* index, const int64_t* layer, const double* weight,
                           ifdtd_probe** out);
int32_t ifdtd_probe_destroy(ifdtd_probe* probe);
int32_t ifdtd_sample(ifdtd_plan* plan, const ifdtd_state* state, const ifdtd_probe* probe,
                     double* out_row, void* stream);
/* Step n_steps times, sampling after every step into out_rows (n_steps, rows)
 * (record_er_observations' inner loop, solver.py:1126-1135). */
int32_t ifdtd_step_sampled(ifdtd_plan* plan, const ifdtd_state* state, const double* currents,
                           int32_t n_steps, const ifdtd_probe* probe, double* out_rows, void* stream);

/* Ensembles.  The reference runs an ensemble as a loop over GeodesicFDTD
 * objects, each calling step() / record_er_observations (solver.py:789-816,
 * 1080-1136); it has no batched runner.  A batch advances all its member plans
 * by the same number of steps: one launch per phase for every group of
 * members whose plans run both phases on the pipeline (grouped by plasma,
 * vertex slot width, copy engine, threads and producer warps), the other
 * members launched on their own within the step, and one launch per step that
 * samples every member's receivers.  Each member's fields come out as from its
 * own ifdtd_step.  All plans share one device and one precision and must
 * outlive the batch; chunk (>= 1) is the steps per captured CUDA graph, capped
 * at the graph_chunk of members launched on their own. */
int32_t ifdtd_batch_create(ifdtd_plan* const* plans, int32_t n_members, int32_t chunk, ifdtd_batch** out);
int32_t ifdtd_batch_destroy(ifdtd_batch* batch);
/* states: n_members states.  currents: device float64 (n_members, n_steps),
 * row i member i's source currents I((n+1/2)dt) (NULL: zero).  probes: NULL or
 * n_members probe handles (entries may be NULL) created on the members' plans;
 * out_rows[i]: device float64 (n_steps, rows_i) for member i's samples. */
int32_t ifdtd_batch_step(ifdtd_batch* batch, const ifdtd_state* states, const double* currents, int32_t n_steps,
                         ifdtd_probe* const* probes, double* const* out_rows, void* stream);
/* Launch layout: batched groups, members launched on their own, and the CTAs
 * of the first group's H and E launches (0 when there is no group). */
int32_t ifdtd_batch_info(const ifdtd_batch* batch, int32_t* groups, int32_t* solo, int32_t* kh_grid,
                         int32_t* ke_grid);

/* Host-side mesh numbering (no device needed): number the distinct pairs
 * (lo[i], hi[i]), 0 <= lo, hi < n_vertices, in order of first appearance, as
 * the reference numbers midpoints and edges while scanning faces in order
 * (mesh.py:569-593, 674-708: a dict assigning len(dict) on first insertion).
 * rank[i] is the number of pair i; first[r] (room for n entries) the position
 * of number r's first appearance; *n_distinct the count of numbers. */
int32_t ifdtd_first_use_numbering(const int64_t* lo, const int64_t* hi, int64_t n, int64_t n_vertices, int64_t* rank,
                                  int64_t* first, int64_t* n_distinct);

/* Host-side grouping (no device needed): order[] receives the permutation that
 * a stable sort of keys[0..n) gives (positions grouped by key, ascending, each
 * group in position order) and counts[k] (room for n_keys entries) the size of
 * group k; every key must lie in [0, n_keys).  It replaces the stable argsort
 * of face corners by vertex behind the plasma coupler's incident-face tables
 * (plasma.py:572-588, a per-vertex list filled while scanning faces in order). */
int32_t ifdtd_stable_group(const int64_t* keys, int64_t n, int64_t n_keys, int64_t* order, int64_t* counts);

/* max |field| of er, et, hr, ht into out4 (device, float64); the four
 * reductions of diagnostics() (solver.py:1027-1030, torch_backend.py:218-219). */
int32_t ifdtd_max_abs(ifdtd_plan* plan, const ifdtd_state* state, double* out4, void* stream);

/* The four topology primitives of the ArrayBackend contract on (N, cols)
 * row-major arrays (backends/base.py:59-73, torch_backend.py:172-198). */
int32_t ifdtd_edge_difference(ifdtd_plan* plan, const void* vertex_values, int32_t cols,
                              void* out, void* stream);
int32_t ifdtd_dual_edge_difference(ifdtd_plan* plan, const void* face_values, int32_t cols,
                                   void* out, void* stream);
int32_t ifdtd_face_circulation(ifdtd_plan* plan, const void* edge_values, int32_t cols,
                               void* out, void* stream);
int32_t ifdtd_dual_cell_circulation(ifdtd_plan* plan, const void* edge_values, int32_t cols,
                                    void* out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* IFDTD_H */
