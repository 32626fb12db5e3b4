"""Learned receiver-trace surrogate, trained on traces the engine generates.

The reference has no surrogate.  A small network maps eight scalars of a run
(ionosphere prefactor sigma0, reference height h0, scale height zeta, ground
conductivity, source latitude and longitude, receiver latitude and longitude)
to the receiver's Er trace.

Network: an MLP (``depth`` SiLU layers of ``width``) and a projection to a
``t0`` x ``c0`` sequence, then non-overlapping 1-D transposed convolutions
(stride = kernel = ``stride``, SiLU between them, per-tap biases) up to
``samples`` outputs.  Activations stay channels-last, so every layer is a
dense product over rows and one GEMM runs all forward and backward products:
``ifdtd_nn_gemm_tc`` (tcgen05.mma on the 5th-generation tensor cores, BF16
inputs, FP32 accumulation in tensor memory) by default, or ``ifdtd_nn_gemm``
(warp-level mma.sync, the same inputs and accumulation) as the checked
alternative (``gemm="mma"``).  Weights
are FP32 masters with BF16 copies; activations between layers are BF16.
Training uses the library's own kernels for every step (GEMMs, bias + SiLU,
its derivative, bias sums, mean-squared error, Adam); PyTorch only holds the
device buffers.

The engine scores the surrogate and is its fallback: ``SurrogateEnsemble`` trains k
networks from different seeds; a case whose members disagree by more than a
threshold (relative spread of their traces) is handed back to the solver.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import _native as N


def _lib():
    return N.load()


def _check(status: int, what: str) -> None:
    N.check(status, what)


@dataclass
class Layer:
    fan_in: int
    fan_out: int
    act: int  # 0 identity, 1 SiLU
    expand: int  # rows of the next layer per row of this one (reshape after the layer)


def architecture(inputs: int = 8, width: int = 512, depth: int = 4, samples: int = 1024, t0: int = 16, c0: int = 64,
                 channels: tuple[int, ...] = (32, 16, 1), stride: int = 4) -> list[Layer]:
    """Layer list of the surrogate; ``samples`` must equal t0 * stride ** len(channels)."""

    if samples != t0 * stride ** len(channels):
        raise ValueError("samples must equal t0 * stride ** len(channels)")
    layers = [Layer(inputs, width, 1, 1)] + [Layer(width, width, 1, 1) for _ in range(depth - 1)]
    layers.append(Layer(width, t0 * c0, 1, t0))
    cin = c0
    for i, cout in enumerate(channels):
        layers.append(Layer(cin, stride * cout, 0 if i == len(channels) - 1 else 1, stride))
        cin = cout
    return layers


GEMM_ENTRIES = {"tcgen05": "ifdtd_nn_gemm_tc_ws", "mma": "ifdtd_nn_gemm"}
WORKSPACE_BYTES = 16 << 20  # split-K partial tiles of the tcgen05 GEMM


class TraceSurrogate:
    """One network with its parameters, Adam state and activation buffers;
    ``gemm`` picks the product kernel ("tcgen05" or "mma")."""

    def __init__(self, layers: list[Layer], *, seed: int = 0, device: str = "cuda", gemm: str = "tcgen05"):
        import torch

        if gemm not in GEMM_ENTRIES:
            raise ValueError(f"gemm must be one of {sorted(GEMM_ENTRIES)}")
        self.gemm_entry = GEMM_ENTRIES[gemm]
        self.torch = torch
        self._workspace = None
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise ValueError("the surrogate kernels run on a CUDA device")
        self.layers = layers
        rng = np.random.default_rng(seed)
        self.w, self.b, self.w16 = [], [], []
        self.mw, self.vw, self.mb, self.vb = [], [], [], []
        for L in layers:
            w = rng.standard_normal((L.fan_out, L.fan_in)) * np.sqrt((2.0 if L.act else 1.0) / L.fan_in)
            self.w.append(torch.tensor(w, dtype=torch.float32, device=self.device))
            self.b.append(torch.zeros(L.fan_out, dtype=torch.float32, device=self.device))
            self.w16.append(self.w[-1].to(torch.bfloat16))
            for lst, shape in ((self.mw, w.shape), (self.vw, w.shape), (self.mb, (L.fan_out,)), (self.vb, (L.fan_out,))):
                lst.append(torch.zeros(shape, dtype=torch.float32, device=self.device))
        self.step_count = 0
        self._acts: list = []

    def _stream(self) -> int:
        return int(self.torch.cuda.current_stream(self.device).cuda_stream)

    def _gemm(self, m, n, k, a, lda, ta, b, ldb, tb, c, ldc) -> None:
        """c = op(a) op(b) with the network's product kernel (bf16 in, fp32 out)."""

        lib, s = _lib(), self._stream()
        if self.gemm_entry == "ifdtd_nn_gemm":
            _check(lib.ifdtd_nn_gemm(m, n, k, a, lda, ta, b, ldb, tb, 1.0, 0.0, c, ldc, s), "ifdtd_nn_gemm")
            return
        if self._workspace is None:
            self._workspace = self.torch.empty(WORKSPACE_BYTES // 4, dtype=self.torch.float32, device=self.device)
        _check(lib.ifdtd_nn_gemm_tc_ws(m, n, k, a, lda, ta, b, ldb, tb, 1.0, 0.0, c, ldc, self._workspace.data_ptr(), WORKSPACE_BYTES, s),
               "ifdtd_nn_gemm_tc_ws")

    def forward(self, x16):
        """x16: (B, inputs) bf16 device tensor -> (B, samples) fp32 predictions."""

        torch = self.torch
        lib, s = _lib(), self._stream()
        rows = int(x16.shape[0])
        self._acts = []
        inp = x16
        z = None
        for i, L in enumerate(self.layers):
            z = torch.empty((rows, L.fan_out), dtype=torch.float32, device=self.device)
            self._gemm(rows, L.fan_out, L.fan_in, inp.data_ptr(), L.fan_in, 0, self.w16[i].data_ptr(), L.fan_in, 1, z.data_ptr(), L.fan_out)
            last = i == len(self.layers) - 1
            y = None if last else torch.empty((rows, L.fan_out), dtype=torch.bfloat16, device=self.device)
            _check(lib.ifdtd_nn_bias_act(rows, L.fan_out, z.data_ptr(), self.b[i].data_ptr(), L.act, None if last else y.data_ptr(), s),
                   "ifdtd_nn_bias_act")
            self._acts.append((inp, z))
            if not last:
                rows *= L.expand
                inp = y.view(rows, L.fan_out // L.expand)
        return z.view(x16.shape[0], -1)

    def backward(self, grad):
        """Gradients of every weight and bias from dLoss/dpred (B, samples) fp32."""

        torch = self.torch
        lib, s = _lib(), self._stream()
        self.gw, self.gb = [None] * len(self.layers), [None] * len(self.layers)
        dy = grad.reshape(self._acts[-1][1].shape).contiguous()
        for i in range(len(self.layers) - 1, -1, -1):
            L = self.layers[i]
            x, z = self._acts[i]
            rows = int(z.shape[0])
            dz = torch.empty_like(z)
            dz16 = torch.empty(z.shape, dtype=torch.bfloat16, device=self.device)
            _check(lib.ifdtd_nn_act_grad(rows, L.fan_out, z.data_ptr(), dy.data_ptr(), L.act, dz.data_ptr(), dz16.data_ptr(), s),
                   "ifdtd_nn_act_grad")
            gw = torch.empty((L.fan_out, L.fan_in), dtype=torch.float32, device=self.device)
            self._gemm(L.fan_out, L.fan_in, rows, dz16.data_ptr(), L.fan_out, 1, x.data_ptr(), L.fan_in, 0, gw.data_ptr(), L.fan_in)
            gb = torch.empty(L.fan_out, dtype=torch.float32, device=self.device)
            _check(lib.ifdtd_nn_col_sum(rows, L.fan_out, dz.data_ptr(), gb.data_ptr(), s), "ifdtd_nn_col_sum")
            self.gw[i], self.gb[i] = gw, gb
            if i > 0:
                dx = torch.empty((rows, L.fan_in), dtype=torch.float32, device=self.device)
                self._gemm(rows, L.fan_in, L.fan_out, dz16.data_ptr(), L.fan_out, 0, self.w16[i].data_ptr(), L.fan_in, 0, dx.data_ptr(),
                           L.fan_in)
                prev = self.layers[i - 1]
                dy = dx.view(rows // prev.expand, prev.fan_out)

    def loss_and_grad(self, pred, target):
        torch = self.torch
        grad = torch.empty_like(pred)
        loss = torch.zeros(1, dtype=torch.float32, device=self.device)
        _check(_lib().ifdtd_nn_mse(int(pred.numel()), pred.data_ptr(), target.data_ptr(), grad.data_ptr(), loss.data_ptr(), self._stream()),
               "ifdtd_nn_mse")
        return loss, grad

    def weighted_loss_and_grad(self, pred, target, row_weight):
        """Squared error with one weight per case (row)."""

        torch = self.torch
        grad = torch.empty_like(pred)
        loss = torch.zeros(1, dtype=torch.float32, device=self.device)
        rows, cols = int(pred.shape[0]), int(pred.shape[1])
        _check(_lib().ifdtd_nn_wmse(rows, cols, pred.data_ptr(), target.data_ptr(), row_weight.data_ptr(), grad.data_ptr(), loss.data_ptr(),
                                    self._stream()), "ifdtd_nn_wmse")
        return loss, grad

    def adam_step(self, lr: float, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8) -> None:
        lib, s = _lib(), self._stream()
        self.step_count += 1
        for i in range(len(self.layers)):
            _check(lib.ifdtd_nn_adam(int(self.w[i].numel()), self.w[i].data_ptr(), self.gw[i].data_ptr(), self.mw[i].data_ptr(),
                                     self.vw[i].data_ptr(), lr, beta1, beta2, eps, self.step_count, self.w16[i].data_ptr(), s), "ifdtd_nn_adam")
            _check(lib.ifdtd_nn_adam(int(self.b[i].numel()), self.b[i].data_ptr(), self.gb[i].data_ptr(), self.mb[i].data_ptr(),
                                     self.vb[i].data_ptr(), lr, beta1, beta2, eps, self.step_count, None, s), "ifdtd_nn_adam")

    def fit(self, x, y, *, iterations: int, batch: int, lr: float = 1e-3, seed: int = 0, lr_final: float | None = None,
            relative: bool = False) -> list[float]:
        """Train on device tensors x (N, inputs) bf16 and y (N, samples) fp32;
        returns the loss of every iteration (one host read at the end).
        relative: weight each case by the inverse mean square of its target, so
        the loss is the cases' mean squared relative error."""

        torch = self.torch
        gen = torch.Generator(device=self.device)
        gen.manual_seed(seed)
        n = int(x.shape[0])
        weight = None
        if relative:
            weight = 1.0 / y.pow(2).mean(dim=1).clamp_min(1e-12 * float(y.pow(2).mean()))
        losses = []
        for it in range(iterations):
            idx = torch.randint(0, n, (min(batch, n),), device=self.device, generator=gen)
            pred = self.forward(x[idx].contiguous())
            if weight is None:
                loss, grad = self.loss_and_grad(pred, y[idx].contiguous())
            else:
                loss, grad = self.weighted_loss_and_grad(pred, y[idx].contiguous(), weight[idx].contiguous())
            self.backward(grad)
            frac = it / max(iterations - 1, 1)
            rate = lr if lr_final is None else lr * (lr_final / lr) ** frac
            self.adam_step(rate)
            losses.append(loss)
        return [float(v) for v in torch.cat(losses).cpu()]

    def predict(self, x, batch: int = 512):
        torch = self.torch
        out = [self.forward(x[i : i + batch].contiguous()).clone() for i in range(0, int(x.shape[0]), batch)]
        return torch.cat(out)


@dataclass
class SurrogateEnsemble:
    """k networks from different seeds; the spread of their predictions decides
    when a case goes back to the solver."""

    members: list[TraceSurrogate] = field(default_factory=list)

    @classmethod
    def train(cls, layers: list[Layer], x, y, *, k: int = 4, iterations: int = 1000, batch: int = 256, lr: float = 1e-3,
              lr_final: float | None = 1e-4, device: str = "cuda", seed: int = 0, relative: bool = False,
              gemm: str = "tcgen05"):
        ens = cls()
        histories = []
        for m in range(k):
            net = TraceSurrogate(layers, seed=seed + 1000 * m, device=device, gemm=gemm)
            histories.append(net.fit(x, y, iterations=iterations, batch=batch, lr=lr, lr_final=lr_final, seed=seed + m,
                                     relative=relative))
            ens.members.append(net)
        return ens, histories

    def predict(self, x):
        """Mean prediction and the relative spread ||std|| / ||mean|| per case."""

        torch = self.torch
        preds = torch.stack([m.predict(x) for m in self.members])
        mean = preds.mean(dim=0)
        spread = preds.std(dim=0, unbiased=False).norm(dim=1) / mean.norm(dim=1).clamp_min(1e-30)
        return mean, spread

    @property
    def torch(self):
        return self.members[0].torch


def relative_l2(pred, target):
    """Per-case ||pred - target|| / ||target||."""

    return (pred - target).norm(dim=1) / target.norm(dim=1).clamp_min(1e-30)


# ----------------------------------------------------------------------------
# Training data from the engine
# ----------------------------------------------------------------------------

FEATURES = ("log10_sigma0", "h0_km", "zeta_km", "log10_ground", "source_lat", "source_lon", "receiver_lat", "receiver_lon")


def encode_features(rows: np.ndarray) -> np.ndarray:
    """Raw (N, 8) parameters -> the network's eight inputs, roughly unit scale:
    log10 sigma0, h0, zeta, log10 ground sigma, the great-circle distance of
    the receiver from the source (in units of 10 degrees), the cosine and sine
    of its bearing, and the sine of the source latitude."""

    r = np.asarray(rows, dtype=np.float64)
    out = np.empty_like(r)
    out[:, 0] = r[:, 0] + 7.0  # log10 sigma0 in [-8, -6]
    out[:, 1] = (r[:, 1] - 62.5) / 7.5  # h0 km in [55, 70]
    out[:, 2] = (r[:, 2] - 4.5) / 1.5  # zeta km in [3, 6]
    out[:, 3] = r[:, 3] + 2.0  # log10 ground in [-3, -1]
    la1, lo1, la2, lo2 = (np.radians(r[:, i]) for i in (4, 5, 6, 7))
    dlon = lo2 - lo1
    cosd = np.sin(la1) * np.sin(la2) + np.cos(la1) * np.cos(la2) * np.cos(dlon)
    out[:, 4] = np.degrees(np.arccos(np.clip(cosd, -1.0, 1.0))) / 10.0
    bearing = np.arctan2(np.sin(dlon) * np.cos(la2), np.cos(la1) * np.sin(la2) - np.sin(la1) * np.cos(la2) * np.cos(dlon))
    out[:, 5] = np.cos(bearing)
    out[:, 6] = np.sin(bearing)
    out[:, 7] = np.sin(la1)
    return out


def _destination(lat_deg: float, lon_deg: float, bearing_deg: float, distance_deg: float) -> tuple[float, float]:
    """Point at ``distance_deg`` along the great circle leaving (lat, lon) at ``bearing_deg``."""

    la, lo, b, d = (np.radians(v) for v in (lat_deg, lon_deg, bearing_deg, distance_deg))
    lat2 = np.arcsin(np.sin(la) * np.cos(d) + np.cos(la) * np.sin(d) * np.cos(b))
    lon2 = lo + np.arctan2(np.sin(b) * np.sin(d) * np.cos(la), np.cos(d) - np.sin(la) * np.sin(lat2))
    return float(np.degrees(lat2)), float((np.degrees(lon2) + 540.0) % 360.0 - 180.0)


def generate_traces(n_runs: int, *, subdivision: int = 6, radial_cells: int = 40, steps: int = 1024, receivers: int = 16,
                    distance_deg: tuple[float, float] = (2.0, 12.0), seed: int = 20260805, batch_members: int = 32,
                    device: str = "cuda", dtype: str = "float32", workers: int | None = None):
    """Run ``n_runs`` seeded members at one mesh level and radial grid through
    ``Ensemble`` and return raw parameters (n_runs * receivers, 8) and surface
    Er traces (n_runs * receivers, steps).  Each member draws sigma0, h0, zeta
    and the ground conductivity as in the ensemble configuration and a source
    vertex at random; its Gaussian source pulse sits inside the window, and its
    receivers lie at random bearings and at great-circle distances within
    ``distance_deg`` of the source, close enough for the pulse to reach them
    within ``steps`` steps.  The draws are made in member order from one seeded
    generator; the members of a batch are then built on ``workers`` host
    threads (default: up to 8), which changes no value."""

    import os
    from concurrent.futures import ThreadPoolExecutor

    from .constants import EPSILON_0
    from .ensemble import Ensemble
    from .materials import EarthIonosphereMaterial
    from .mesh import build_geodesic_mesh
    from .solver import GeodesicFDTD, SimulationConfig
    from .sources import GaussianCurrent, geographic_distribution
    from .workloads import vertex_lat_lon

    rng = np.random.default_rng(seed)
    mesh = build_geodesic_mesh(subdivision)
    cfg = SimulationConfig(subdivision=subdivision, radial_cells=radial_cells)
    # the time step depends on the mesh and radial grid only, so one material-free
    # run gives the window that places every source pulse
    window = steps * GeodesicFDTD(cfg, mesh=mesh, device=device, dtype=dtype).time_step_s
    workers = workers or max(1, min(8, os.cpu_count() or 1))

    def build(draw):
        sigma0, h0, zeta, ground, lat, lon, bearings, distances = draw
        material = EarthIonosphereMaterial(lithosphere_conductivity_s_m=ground, ionosphere_reference_height_m=h0,
                                           ionosphere_scale_height_m=zeta, ionosphere_prefactor_hz=sigma0 / EPSILON_0)
        source = GaussianCurrent(latitude_deg=lat, longitude_deg=lon, peak_current_a=1.0e6, carrier_frequency_hz=0.0,
                                 center_time_s=0.35 * window, one_over_e_half_width_s=0.12 * window)
        sim = GeodesicFDTD(cfg, material=material, source=source, mesh=mesh, device=device, dtype=dtype)
        rows, supports = [], []
        for b, d in zip(bearings, distances):
            rlat, rlon = _destination(lat, lon, b, d)
            supports.append(geographic_distribution(sim, rlat, rlon, 0.0))
            rows.append((np.log10(sigma0), h0 / 1e3, zeta / 1e3, np.log10(ground), lat, lon, rlat, rlon))
        v = np.stack([r[0] for r in supports]).astype(np.int64)
        k = np.asarray([r[1] for r in supports], dtype=np.int64)
        w = np.stack([r[2] for r in supports])
        return sim, (v, k, w), rows

    params, traces = [], []
    with ThreadPoolExecutor(max_workers=workers) as pool:
        for start in range(0, n_runs, batch_members):
            draws = []
            for _ in range(min(batch_members, n_runs - start)):
                sigma0 = 10.0 ** rng.uniform(-8.0, -6.0)
                h0 = rng.uniform(55_000.0, 70_000.0)
                zeta = rng.uniform(3_000.0, 6_000.0)
                ground = 10.0 ** rng.uniform(-3.0, -1.0)
                lat, lon = vertex_lat_lon(mesh.vertices, int(rng.integers(mesh.n_vertices)))
                bearings = rng.uniform(0.0, 360.0, receivers)
                distances = rng.uniform(distance_deg[0], distance_deg[1], receivers)
                draws.append((sigma0, h0, zeta, ground, lat, lon, bearings, distances))
            built = list(pool.map(build, draws))
            sims = [b[0] for b in built]
            with Ensemble(sims) as ens:
                out = ens.record_er_observations([b[1] for b in built], steps)
            for t in out:
                traces.append(np.asarray(t[1:], dtype=np.float64).T)  # (receivers, steps)
            for b in built:
                params.extend(b[2])
            del sims, built
    return np.asarray(params, dtype=np.float64), np.concatenate(traces, axis=0)


def gemm_throughput(m: int, n: int, k: int, *, gemm: str = "tcgen05", reps: int = 20, device: str = "cuda") -> dict:
    """Time one surrogate GEMM shape (bf16 inputs, fp32 output, C = A B^T as the
    forward pass calls it) with CUDA events on the current stream: median
    milliseconds per call over ``reps`` calls after three warm-up calls, the
    TFLOP/s of 2 m n k, and the relative error against a float32 product."""

    import statistics

    import torch

    if gemm not in GEMM_ENTRIES:
        raise ValueError(f"gemm must be one of {sorted(GEMM_ENTRIES)}")
    lib = _lib()
    g = torch.Generator(device=device).manual_seed(m + 3 * n + 7 * k)
    a = torch.randn((m, k), device=device, generator=g).to(torch.bfloat16)
    b = torch.randn((n, k), device=device, generator=g).to(torch.bfloat16)
    c = torch.empty((m, n), device=device, dtype=torch.float32)
    s = int(torch.cuda.current_stream(device).cuda_stream)

    ws = torch.empty(WORKSPACE_BYTES // 4, dtype=torch.float32, device=device)

    def call():
        if gemm == "mma":
            _check(lib.ifdtd_nn_gemm(m, n, k, a.data_ptr(), k, 0, b.data_ptr(), k, 1, 1.0, 0.0, c.data_ptr(), n, s), "ifdtd_nn_gemm")
        else:
            _check(lib.ifdtd_nn_gemm_tc_ws(m, n, k, a.data_ptr(), k, 0, b.data_ptr(), k, 1, 1.0, 0.0, c.data_ptr(), n, ws.data_ptr(),
                                           WORKSPACE_BYTES, s), "ifdtd_nn_gemm_tc_ws")

    for _ in range(3):
        call()
    marks = [torch.cuda.Event(enable_timing=True) for _ in range(reps + 1)]
    marks[0].record()
    for i in range(reps):
        call()
        marks[i + 1].record()
    torch.cuda.synchronize()
    ms = statistics.median(marks[i].elapsed_time(marks[i + 1]) for i in range(reps))
    ref = a.float() @ b.float().T
    err = float((c - ref).norm() / ref.norm())
    return {"m": m, "n": n, "k": k, "gemm": gemm, "ms": ms, "tflops": 2.0 * m * n * k / (ms / 1e3) / 1e12, "rel_err": err}


if __name__ == "__main__":
    import json
    import sys

    # python -m ionosphere_fdtd_b200.surrogate M N K [tcgen05|mma]: one GEMM timing line
    shape = [int(v) for v in sys.argv[1:4]] if len(sys.argv) >= 4 else [4096, 4096, 4096]
    kind = sys.argv[4] if len(sys.argv) >= 5 else "tcgen05"
    print(json.dumps(gemm_throughput(*shape, gemm=kind)))
