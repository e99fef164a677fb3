"""Benchmark of the unsplit hydro step (zone-updates/s).

Workload: 3D Kelvin-Helmholtz, 512^3 cells as 64^3 blocks of 8^3 interior
cells (FLASH's 4 guard layers are filled inside the kernels), gamma = 5/3,
periodic boundaries, PPM with characteristic limiting and flattening, CFL
0.8, the time step recomputed every step (Hydro_computeDt reduction +
Driver_computeDt growth limit).  Inputs are synthetic (seeded noise, numpy
PCG64 seed 12345).

One step = the device pass of the hot path over all blocks (k_sig + one
fused kernel per direction) plus the CFL reduction read back to the host.
Paths (all replay the dt sequence of the first):
  fp64           plain FP64 HLLC (bit-identical to the CPU oracle)
  fp64_exact     FP64 with the exact Riemann solver (FP64 reference of the
                 exact-solver paths)
  mixed          FP32 reconstruction, FP64 HLLC and update
  mixed_exact    FP32 reconstruction, FP64 exact solver and update
  mixed_learned  as mixed_exact, Newton started from the tensor-core MLP
                 guess trained on this run's harvested face states
``value`` is the last path (by default mixed_learned, the metric's
"batched mixed+learned") with the state resident in HBM; each path's error
is measured on the device against its FP64 reference on the same run.
``e2e`` is the same metric through the C-ABI with host UNK buffers
(interior-only FLASH UNK, 11 variables, pinned): upload, step, dt, download
every step.  The default line also carries the batched AMR workload
(``amr``: 2D four-quadrant hierarchy of 19,456 leaf blocks) and the
isolated exact-Riemann workload (``riemann``: 1e8 interface pairs; the
learned start with the network on the tcgen05 tensor cores and per warp on
mma.sync, beside the two-rarefaction start).

``--impl reference`` times the CPU oracle (the C restatement of the
reference's Fortran; the Fortran itself cannot be built here) with all host
threads on a bounded sample of the same workload: a window of 8^3 blocks
(64^3 zones) of the 512^3 grid with its initial data, advanced with
FLASH's own method (PPM + HLLC) from guard cells of the surrounding blocks.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "zone-updates/s on 1 B200: batched mixed+learned vs plain FP64, rel L1<=1e-6"
UNIT = "zone-updates/s"
BYTES_PER_ZONE = 80.0          # read + write of 5 FP64 state variables
# DRAM bytes per zone-update of one step (k_sig + the three direction
# kernels) from ncu captures of the 160^3 KH step (dram__bytes_read.sum +
# dram__bytes_write.sum over 4.096e6 zones), scaled to the workload by its
# zone count (traffic grows in proportion)
TRAFFIC_PER_ZONE = {"fp64": 1250.6, "mixed": 864.4, "mixed_exact": 893.5, "mixed_learned": 893.5}
# Floating-point operations per zone-update of one step (k_sig + the three
# direction kernels), counted by ncu on the same 160^3 KH step:
# smsp__sass_thread_inst_executed_op_{dadd,dmul,dfma,fadd,fmul,ffma}_pred_on
# (an FMA counts two), divided by the zones; and the FP64 pipe utilisation
# (sm__pipe_fp64_cycles_active, % of peak over the kernels' active cycles,
# weighted by their durations).
FLOPS_PER_ZONE = {"fp64": {"f64": 7626, "f32": 394, "fp64_pipe_pct": 27.1},
                  "mixed": {"f64": 1192, "f32": 1984, "fp64_pipe_pct": 15.3},
                  "mixed_exact": {"f64": 2120, "f32": 2035, "fp64_pipe_pct": 19.6},
                  "mixed_learned": {"f64": 2120, "f32": 2035, "fp64_pipe_pct": 19.6}}
# nominal vector peaks of a B200 at the 1965 MHz maximum SM clock: 148 SMs x
# 64 FP64 (128 FP32) FMA lanes x 2 flops; no measured FP64/FP32 peak exists
# for this pool, so the compute fractions are "of nominal"
FP64_PEAK_TFLOPS = 148 * 64 * 2 * 1.965e9 / 1e12
FP32_PEAK_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def measured_bf16_peak():
    """Dense BF16 tensor throughput (TFLOP/s) for a kernel timed alone: the
    measured burst figure, else the fallback."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        if "bf16_tflops" in d:
            return float(d["bf16_tflops"]), "measured"
    return 1590.0, "fallback"


def riemann_roofline(n, solve_ms, network_ms):
    """Rooflines of the isolated workload: the learned solve against HBM
    (7 FP64 in, p* and u* and two flag bytes out per pair), the network
    alone against the BF16 tensor peak (the three MMAs of a 128-row tile,
    K and N padding included: 2 (16 x 64 + 80 x 64 + 64 x 16) FLOP per
    row)."""
    hbm, hbm_kind = measured_peaks()
    tc, tc_kind = measured_bf16_peak()
    bpp = 7 * 8 + 2 * 8 + 2
    fpp = 2 * (16 * 64 + 80 * 64 + 64 * 16)
    rows = -(-n // 128) * 128
    gbs = n * bpp / (solve_ms * 1e-3) / 1e9
    tfs = rows * fpp / (network_ms * 1e-3) / 1e12
    return {"solve": {"bound": "issue (FP64 set-up and Newton)", "hbm_bytes_per_pair": bpp, "achieved_gbs": gbs,
                      "peak_gbs": hbm, "frac": gbs / hbm, "peak_kind": hbm_kind},
            "network_alone": {"tensor_flops_per_pair": fpp, "achieved_tflops": tfs, "peak_tflops": tc,
                              "frac": tfs / tc, "peak_kind": tc_kind,
                              "note": "tcgen05 kind::f16, BF16 operands, FP32 accumulator; the time includes "
                                      "the per-pair FP64 set-up and features"}}


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def pin_openmp():
    """OpenMP settings of the CPU oracle: one thread per host core the
    process may use, bound to cores (read when the oracle library's OpenMP
    runtime starts, i.e. before its first parallel region)."""
    os.environ.setdefault("OMP_NUM_THREADS", str(host_cores()))
    os.environ.setdefault("OMP_PROC_BIND", "close")
    os.environ.setdefault("OMP_PLACES", "cores")


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(5)
            except Exception:
                self.p.kill()

    def summary(self):
        self.f.flush()
        rows = []
        with open(self.f.name) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        load = [s for s in sm if s > 500] or sm
        return {"sm_mhz": float(np.median(load)) if load else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def kh_workload(nblk=64, nguard=0, nspecies=0, nmass_scalars=0):
    from flash5_b200 import abi, setups
    from flash5_b200.grid import UniformGrid
    g = UniformGrid(3, (8, 8, 8), (nblk, nblk, nblk), bc="periodic", nguard=nguard, nspecies=nspecies,
                    nmass_scalars=nmass_scalars)
    unk = setups.add_species(g, setups.kelvin_helmholtz(g))
    return g, unk, abi


def kh_config(args, world=1, riemann="exact (Newton 1e-12)", head="mixed_learned"):
    """The workload description shared by both arms of the benchmark."""
    zones = 512 * args.nblk ** 3
    return {"workload": f"3D Kelvin-Helmholtz {8 * args.nblk}^3 as {args.nblk}^3 blocks of 8^3 (+4 guard "
                        "filled in-kernel), gamma 5/3, periodic, PPM, CFL 0.8, dt from the CFL reduction "
                        "every step" + (f", {world} such boxes stacked along z (periodic), blocks sharded "
                                        "over the ranks in Morton order, ghost blocks exchanged by NCCL "
                                        "point-to-point every step, NCCL dt min" if world > 1 else ""),
            "riemann": riemann, "zones_per_gpu": zones,
            "l2": f"inputs larger than L2 (state {zones * 40 / 1e6:.0f} MB)",
            **({"species": args.nspecies, "mass_scalars": args.nmass_scalars,
                "species_note": "dense-layer species pair and passive tracers; species pass in FP64 on the FP64 "
                                "paths, FP32 face values with FP64 fluxes and update on the mixed paths"}
               if args.nspecies + args.nmass_scalars else {}),
            "path": head}


def run_device(h, steps, warmup, dts=None, sampler=None, dist=None):
    """Time `steps` hydro steps with the state resident on the device.
    Returns (ms_per_step, dt list, launches per step)."""
    import torch
    from flash5_b200.hydro import next_dt
    stream = torch.cuda.ExternalStream(h.stream)
    dt, _ = h.compute_dt()
    if dist is not None:
        dt = dist_min(dist, dt)
    dt_old = dt
    used = []
    t = 0.0

    def one(i):
        nonlocal dt, dt_old, t
        d = dts[i] if dts is not None else dt
        h(t + d, d, dt_old)
        used.append(d)
        t += d
        dcfl, _ = h.compute_dt()
        if dist is not None:
            dcfl = dist_min(dist, dcfl)
        dt_old, dt = d, next_dt(dcfl, d)

    for i in range(warmup):
        one(i)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ctx = sampler if sampler is not None else _null()
    with ctx:
        e0.record(stream)
        for i in range(warmup, warmup + steps):
            one(i)
        e1.record(stream)
        e1.synchronize()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    ms = e0.elapsed_time(e1) / steps
    return ms, used, h.last_launch_count + 1


class _null:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        pass


def dist_min(dist, x):
    import torch
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MIN)
    return float(t.item())


def dist_max(dist, x):
    import torch
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_e2e(h, unk_host, steps, warmup):
    """upload -> step -> dt -> download per step through the C-ABI, host buffers."""
    import torch
    from flash5_b200.hydro import next_dt
    stream = torch.cuda.ExternalStream(h.stream)
    h.upload(unk_host)
    dt, _ = h.compute_dt()
    dt_old, t = dt, 0.0

    def one():
        nonlocal dt, dt_old, t
        h.upload(unk_host)
        h(t + dt, dt, dt_old)
        dcfl, _ = h.compute_dt()
        h.download(unk_host)
        t += dt
        dt_old, dt = dt, next_dt(dcfl, dt)

    for _ in range(warmup):
        one()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        one()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / steps


def e2e_guard_inclusive(params, weights, dev, nblk=32, steps=3, warmup=2):
    """e2e with FLASH's own guard-inclusive UNK, unk(var, 1:16, 1:16, 1:16,
    blk) for 8^3 blocks (NGUARD = 4), as the ISO_C_BINDING shim passes it:
    KH 256^3, the same path; the transfers move the interiors only."""
    import torch
    from flash5_b200.hydro import Hydro
    g, unk, _ = kh_workload(nblk, nguard=4)
    h = Hydro(params, g, device=dev)
    if weights is not None:
        h.set_guess_weights(weights)
    pinned = torch.empty(unk.shape, dtype=torch.float64, pin_memory=True)
    host = pinned.numpy()
    host[...] = unk
    del unk
    ms = run_e2e(h, host, steps, warmup)
    h.close()
    zones = g.ncells
    return {"value": zones / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms, "zones": zones,
            "host_unk_bytes": host.nbytes, "h2d_bytes_per_step": 6 * 8 * zones, "d2h_bytes_per_step": 5 * 8 * zones,
            "workload": f"3D Kelvin-Helmholtz {8 * nblk}^3, guard-inclusive FLASH UNK (16^3 cells per 8^3 block, "
                        "11 vars), pinned host memory, same path as the headline"}


def device_errors(a, b):
    """Error norms of state a against state b ([5, n] device tensors of
    dens, velx, vely, velz, eint): per conserved variable (rho, rho u, rho v,
    rho w, rho E) sfocu's L1 relative norm with each variable's own norm,
    the magnitude error max|a-b| / max|b|, and the L1 norm with the momentum
    components normalised by the momentum vector's norm sum |rho v|."""
    import torch

    def cons(s):
        r = s[0]
        ek = 0.5 * (s[1] * s[1] + s[2] * s[2] + s[3] * s[3])
        return {"dens": r, "xmom": r * s[1], "ymom": r * s[2], "zmom": r * s[3], "ener": r * (s[4] + ek)}
    ca, cb = cons(a), cons(b)
    l1, linf, l1v = {}, {}, {}
    mag = torch.sqrt(cb["xmom"] ** 2 + cb["ymom"] ** 2 + cb["zmom"] ** 2).sum().item()
    for k in ca:
        d = (ca[k] - cb[k]).abs()
        den = cb[k].abs().sum().item()
        l1[k] = d.sum().item() / den if den > 0 else d.sum().item()
        mx = cb[k].abs().max().item()
        linf[k] = d.max().item() / mx if mx > 0 else d.max().item()
        l1v[k] = l1[k] if k in ("dens", "ener") else d.sum().item() / mag
    return l1, linf, l1v


# ---------------------------------------------------------------------------
# CPU oracle legs (the checker's C restatement; only these legs run it)
# ---------------------------------------------------------------------------
def kh_window(nblk, w=8):
    """A window of w^3 blocks of the nblk^3-block KH grid (straddling the
    shear interface at y = 0.25) plus the ring of blocks around it, with the
    full grid's initial data: (local grid, UNK, owned local indices)."""
    from flash5_b200 import setups
    from flash5_b200.shard import LocalGrid
    lo = (0, max(0, nblk // 4 - w // 2), 0)
    w = min(w, nblk)
    own = [(lo[0] + i, lo[1] + j, lo[2] + k) for k in range(w) for j in range(w) for i in range(w)]
    ring = set()
    if w < nblk:
        for (i, j, k) in own:
            for dk in (-1, 0, 1):
                for dj in (-1, 0, 1):
                    for di in (-1, 0, 1):
                        c = ((i + di) % nblk, (j + dj) % nblk, (k + dk) % nblk)
                        ring.add(c)
        ring -= set(own)
    coords = own + sorted(ring)
    g = LocalGrid(3, (8, 8, 8), (nblk, nblk, nblk), coords, bc="periodic")
    unk = setups.kelvin_helmholtz(g)
    return g, unk, np.arange(len(own), dtype=np.int32)


def cpu_sample(nblk, steps=None, warmup=3, seconds=10.0):
    """The oracle (C restatement of the reference, FLASH's method PPM + HLLC,
    OpenMP over blocks on all host cores) advancing a 64^3-zone window of the
    benchmark grid: per-step times after `warmup` steps, either `steps`
    steps or as many as fit in `seconds`; the median step sets the rate."""
    pin_openmp()
    from flash5_b200 import abi
    from flash5_b200.hydro import next_dt
    from oracle import orc
    g, unk, owned = kh_window(nblk)
    p = abi.default_params(gamma=5.0 / 3.0)
    o = orc.Oracle(p, g)
    o.eos_init(unk)
    _, dt, _ = o.compute_dt(unk)
    dt_old, t = dt, 0.0

    def one():
        nonlocal dt, dt_old, t
        o.hydro(unk, t + dt, dt, dt_old, blocks=owned)
        _, dcfl, _ = o.compute_dt(unk)
        t += dt
        dt_old, dt = dt, next_dt(dcfl, dt)

    for _ in range(warmup):
        one()
    times = []
    t0 = time.perf_counter()
    while (steps is None and (len(times) < 3 or time.perf_counter() - t0 < seconds)) or \
            (steps is not None and len(times) < steps):
        s = time.perf_counter()
        one()
        times.append(time.perf_counter() - s)
    zones = len(owned) * 512
    med = float(np.median(times))
    return {"value": zones / med, "unit": UNIT, "cores": int(os.environ["OMP_NUM_THREADS"]), "kind": "port",
            "sample": f"oracle C port (FLASH's PPM + HLLC, FP64), OpenMP on {os.environ['OMP_NUM_THREADS']} "
                      f"cores bound close: a 64^3-zone window (512 blocks of 8^3, straddling the shear "
                      f"interface) of the {8 * nblk}^3 grid with its initial data, guard cells from the "
                      f"surrounding blocks; median of {len(times)} steps after {warmup} warm-up steps "
                      f"(mean {np.mean(times) * 1e3:.1f} ms, min {np.min(times) * 1e3:.1f} ms, "
                      f"max {np.max(times) * 1e3:.1f} ms per step)",
            "why_window": f"at this rate one step of the whole {8 * nblk}^3 grid would take "
                          f"{(8 * nblk) ** 3 * med / zones:.0f} s on these cores, and the run's warm-up and timed "
                          f"steps {(8 * nblk) ** 3 * med / zones * (warmup + (steps or 3)) / 60:.0f} min; the "
                          f"window keeps the grid's data, method and per-zone work",
            "ms_per_step_median": med * 1e3}


def amr_cpu_baseline(seconds=10.0):
    """Oracle AMR step on a 16x16-root, 3-level four-quadrant hierarchy
    (same refinement rule), all host threads."""
    pin_openmp()
    from flash5_b200 import abi, setups
    from flash5_b200.amr import four_quadrant_hierarchy
    from flash5_b200.hydro import next_dt
    from oracle import orc
    g = four_quadrant_hierarchy(nblk=16, max_level=3)
    p = abi.default_params()
    unk = setups.four_quadrant(g)
    o = orc.Oracle(p, g)
    o.eos_init(unk)
    _, dt, _ = o.compute_dt(unk)
    times = []
    t0 = time.perf_counter()
    while len(times) < 3 or time.perf_counter() - t0 < seconds:
        s = time.perf_counter()
        o.hydro(unk, dt, dt, dt)
        _, dcfl, _ = o.compute_dt(unk)
        dt = next_dt(dcfl, dt)
        times.append(time.perf_counter() - s)
    med = float(np.median(times))
    return {"value": g.ncells / med, "unit": UNIT, "cores": int(os.environ["OMP_NUM_THREADS"]), "kind": "port",
            "sample": f"2D four-quadrant AMR, 16^2 root blocks, 3 levels, {g.nleaves} leaves, median of "
                      f"{len(times)} steps, oracle C port, OpenMP"}


# ---------------------------------------------------------------------------
# learned guess
# ---------------------------------------------------------------------------
def train_guess(g, unk, abi, dev, dts, gamma=5.0 / 3.0):
    """Learned star-pressure guess for the hydro faces: run two steps of the
    mixed exact-solver path with face-state harvesting on (the faces where
    the network is consulted: strong waves, inexact two-rarefaction guess),
    top the sample up with the solver's own isolated solves when the flow
    has few such faces, and train the network with the library's training
    kernels.  Returns the FP32 weights (outside the timed region)."""
    import torch
    from flash5_b200.hydro import Hydro
    from flash5_b200.riemann import ExactRiemann
    t0 = time.perf_counter()
    h = Hydro(abi.default_params(gamma=gamma, precision=abi.PREC_MIXED, riemann_solver=abi.RS_EXACT), g,
              device=dev)
    h.upload(unk)
    dt, _ = h.compute_dt()
    h.harvest(2_000_000, keep_log2=0)
    t = 0.0
    for i in range(2):
        d = dts[i] if dts is not None else dt
        h(t + d, d, d)
        t += d
    S = h.harvest_fetch(torch)
    h.close()
    r = ExactRiemann(dev)
    nh = int(S.shape[1])
    if nh < 1_000_000:
        S = torch.cat([S, r.generate(7, 1_000_000 - nh)], dim=1).contiguous()
    loss, ns = r.fit(S, epochs=8, batch=4096, lr=2e-3)
    w = r.weights()
    r.close()
    return w, {"hydro_face_states": nh, "isolated_states": int(S.shape[1]) - nh, "samples": ns, "epochs": 8,
               "final_mse": loss, "seconds": time.perf_counter() - t0,
               "source": "2 steps of the mixed exact path (faces with strong waves), topped up with isolated "
                         "solves of the 1e8-pair distribution"}


# ---------------------------------------------------------------------------
# isolated Riemann workload
# ---------------------------------------------------------------------------
def riemann_run(args, n=None, steps=None, warmup=None):
    """Isolated exact Riemann solves (1e8 interface pairs): two-rarefaction
    guess vs the learned guess trained on solver-harvested states."""
    import torch
    from flash5_b200.riemann import INFER_TCGEN05, INFER_WARP_MMA, ExactRiemann
    torch.cuda.set_device(0)
    n = n or args.riemann_n
    steps = steps or args.steps
    warmup = warmup or args.warmup
    r = ExactRiemann(0)
    stream = r.stream
    # training set harvested from the solver's own solves of another seed
    Str = r.generate(1, args.riemann_train_n)
    otr, _, _ = r.solve(Str, learned=False)
    X, T, ns = r.make_samples(Str, otr)
    t0 = time.perf_counter()
    loss = r.train(X, T, ns, epochs=args.riemann_epochs, batch=4096, lr=2e-3)
    train_s = time.perf_counter() - t0
    del Str, otr, X, T
    S = r.generate(20251203, n)
    out = r.empty(2, n)
    its = r.empty(n, dtype=torch.uint8)
    flg = r.empty(n, dtype=torch.uint8)
    res = {}
    # learned: the network on the tcgen05 tensor cores (the default);
    # learned_warp_mma: the same network per warp on mma.sync
    for name, learned, mode in (("two_rarefaction", False, INFER_TCGEN05), ("learned", True, INFER_TCGEN05),
                                ("learned_warp_mma", True, INFER_WARP_MMA)):
        r.set_inference(mode)
        for _ in range(max(1, warmup)):
            r.solve(S, learned, out=out, iters=its, flags=flg)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            r.solve(S, learned, out=out, iters=its, flags=flg)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / steps
        it = its.cpu().numpy()
        fl = flg.cpu().numpy()
        ok = (fl & 2) == 0
        hist = np.bincount(it[ok], minlength=12)[:12].tolist()
        res[name] = {
            "solves_per_s": n / (ms * 1e-3), "ms": ms, "mean_iters": float(it[ok].mean()), "iter_hist": hist,
            "fallback_frac": float(((fl & 1) != 0)[ok].mean()), "nonconverged": int(((fl & 4) != 0).sum()),
            "vacuum": int((~ok).sum()), "pstar": out[0].clone(), "_it": it, "_fl": fl}
    r.set_inference(INFER_TCGEN05)
    assert r.sync() == 0
    # where the network was consulted (strong waves, inexact two-rarefaction
    # guess): evaluations of both starts on those solves
    cons = (res["learned"]["_fl"] & 8) != 0
    for k in res:
        it = res[k].pop("_it")
        res[k].pop("_fl")
        res[k]["mean_iters_where_consulted"] = float(it[cons].mean()) if cons.any() else None
    consulted_frac = float(cons.mean())
    # the network alone, dense over every pair: features + 8-64-64-1 BF16
    # inference (what the learned start costs per consulted solve at best),
    # on the tcgen05 tensor cores and per warp on mma.sync
    predict_ms = {}
    for name, mode in (("tcgen05", INFER_TCGEN05), ("warp_mma", INFER_WARP_MMA)):
        r.set_inference(mode)
        for _ in range(max(1, warmup)):
            yv = r.predict(S)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            yv = r.predict(S)
        e1.record(stream)
        e1.synchronize()
        predict_ms[name] = e0.elapsed_time(e1) / steps
        del yv
    r.set_inference(INFER_TCGEN05)
    p0, p1, p2 = (res[k].pop("pstar") for k in ("two_rarefaction", "learned", "learned_warp_mma"))
    okd = torch.tensor(ok, device=p0.device)
    rel = max(((p - p0).abs() / p0.clamp_min(1e-300))[okd].max().item() for p in (p1, p2))
    r.close()
    del S, out, its, flg, p0, p1
    torch.cuda.empty_cache()
    return {"metric": "exact Riemann star-pressure solves/s (Newton to 1e-12, FP64)",
            "value": res["learned"]["solves_per_s"], "unit": "solves/s", "n_gpus": 1, "steps": steps,
            "warmup": warmup, "ms_per_step": res["learned"]["ms"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64 Newton, bf16 MLP (f32 acc)",
            "data": "synthetic (splitmix64 seed 20251203)",
            "config": {"workload": f"{n:.0e} isolated interface pairs: p ratio log-uniform 1e-4..1e4, rho ratio "
                                   "1e-3..1e3, u uniform +-5 c, gamma in {1.4, 5/3}; MLP 8-64-64-1 BF16 on tcgen05 "
                                   "tensor cores (TMEM accumulator, 128 interfaces per MMA tile)"},
            "paths": res, "speedup_vs_two_rarefaction": res["two_rarefaction"]["ms"] / res["learned"]["ms"],
            "max_rel_pstar_diff_learned_vs_tr": rel, "consulted_frac": consulted_frac,
            "network_dense_ms": predict_ms,
            "roofline": riemann_roofline(n, res["learned"]["ms"], predict_ms["tcgen05"]),
            "network_dense_note": "the network over every pair (features + tensor-core MLP, written out), tcgen05 "
                                  "and per-warp mma.sync: its own cost per solve, against the Newton evaluations it "
                                  "saves where consulted",
            "training": {"samples": ns, "epochs": args.riemann_epochs, "final_mse": loss, "seconds": train_s}}


# ---------------------------------------------------------------------------
# batched AMR workload
# ---------------------------------------------------------------------------
def amr_run(args, paths, e2e=True, regrid=True, cpu=True, steps=None, warmup=None):
    """Batched AMR hierarchy, 2D four-quadrant Riemann problem: 4 levels,
    19,456 leaf blocks of 16^2 refined where a seeded smoothed density
    gradient is large; every level advanced in one graph-replayed step with
    one dt, fine/coarse flux correction on.  Returns the JSON line."""
    import torch
    from flash5_b200 import abi, setups
    from flash5_b200.amr import four_quadrant_hierarchy
    from flash5_b200.hydro import Hydro
    torch.cuda.set_device(0)
    steps = steps or args.steps
    warmup = warmup or args.warmup
    t0 = time.perf_counter()
    g = four_quadrant_hierarchy(nblk=args.amr_nblk)
    unk = setups.four_quadrant(g)
    build_s = time.perf_counter() - t0
    zones = g.ncells
    peak, peak_kind = measured_peaks()
    ms, outs, dts, launches, clocks, e2e_ms = {}, {}, None, {}, None, None
    tunings = {}
    regrid_info = None
    # (precision, Riemann solver, the FP64 path the errors are measured against, learned guess)
    spec = {"fp64": (abi.PREC_FP64, abi.RS_HLLC, None, 0), "fp64_exact": (abi.PREC_FP64, abi.RS_EXACT, None, 0),
            "mixed": (abi.PREC_MIXED, abi.RS_HLLC, "fp64", 0),
            "mixed_exact": (abi.PREC_MIXED, abi.RS_EXACT, "fp64_exact", 0),
            "mixed_learned": (abi.PREC_MIXED, abi.RS_EXACT, "fp64_exact", 1)}
    paths = [p for p in paths if p in spec] or ["fp64", "mixed"]
    training = None
    leaves = torch.tensor(g.leaf_ids, dtype=torch.long, device="cuda")
    ncb = 16 * 16
    lidx = (leaves[:, None] * ncb + torch.arange(ncb, device="cuda")[None, :]).reshape(-1)
    for name in paths:
        pr, rsv, _, learned = spec[name]
        h = Hydro(abi.default_params(precision=pr, riemann_solver=rsv, learned_guess=learned), g)
        if learned:
            weights, training = train_guess(g, unk, abi, 0, dts, gamma=abi.default_params().gamma)
            h.set_guess_weights(weights)
        h.upload(unk)
        if not args.no_tune:
            best, trials = h.autotune(dts[0] if dts is not None else h.compute_dt()[0], steps=2)
            tunings[name] = {"best": best, "trials_ms": {"/".join(str(v) for v in t.values()): round(m, 4)
                                                         for t, m in trials},
                             "trial_key": "sig_threads/dir_threads/mx_threads/mx_runs/mx_sweep"}
        headline = name == paths[-1]
        sampler = ClockSampler(0) if headline else None
        ms[name], used, launches[name] = run_device(h, steps, warmup, dts=dts, sampler=sampler)
        if dts is None:
            dts = used
        if headline:
            clocks = sampler.summary()
        outs[name] = h.export_state(torch)[:, lidx]
        if headline and e2e:
            pinned = torch.empty(unk.shape, dtype=torch.float64, pin_memory=True)
            host = pinned.numpy()
            host[...] = unk
            e2e_ms = run_e2e(h, host, max(3, min(steps, 8)), 3)
        if headline and regrid:
            # one refinement cycle on the stepped state: the estimator of
            # dens and pres on every node (device), marks and new tree
            # (host), data of the new tree (device)
            from flash5_b200.amr import update_refinement
            est = []
            for _ in range(3):
                t1 = time.perf_counter()
                h.estimate_error("pres", 0.01)
                est.append(time.perf_counter() - t1)
            tm = {}
            h, g_new = update_refinement(h, g, ("dens", "pres"), 0.8, 0.2, 0.01, timings=tm)
            regrid_info = {"estimate_one_var_ms": 1e3 * min(est), "nodes": g.nblocks,
                           "cycle": {k: (round(v * 1e3, 3) if k.endswith("_s") else v) for k, v in tm.items()},
                           "cycle_units": "ms (mark_and_tree: estimator of dens + pres, marks and new tree, all on "
                                          "the device; grid: host descriptors of the new tree; data: new context + "
                                          "device regrid)",
                           "new_leaves": int(g_new.nleaves), "old_leaves": int(g.nleaves),
                           "cutoffs": {"refine": 0.8, "derefine": 0.2, "filter": 0.01}}
        h.close()
    head = paths[-1]
    ref_of = {n: spec[n][2] for n in outs if spec[n][2] in outs}
    errs = {n: device_errors(outs[n], outs[r]) for n, r in ref_of.items()}
    outs.clear()
    cpu_r = amr_cpu_baseline() if cpu else None
    achieved = zones * BYTES_PER_ZONE / (ms[head] * 1e-3) / 1e9
    levels = np.bincount(g.levels[g.is_leaf], minlength=g.max_level + 1)[1:].tolist()
    line = {
        "metric": METRIC, "value": zones / (ms[head] * 1e-3), "unit": UNIT, "n_gpus": 1, "steps": steps,
        "warmup": warmup, "ms_per_step": ms[head], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None,
        "dtype": ("f32 reconstruction, f64 Riemann/update" + (", bf16 MLP guess" if head == "mixed_learned" else ""))
                 if head.startswith("mixed") else "f64",
        "data": "synthetic (four-quadrant states; hierarchy from a seeded smoothed density, PCG64 seed 2024)",
        "config": {"workload": f"2D four-quadrant Riemann problem on a {g.max_level}-level AMR hierarchy, "
                               f"{g.nleaves} leaf blocks of 16^2 + 4 guard ({levels} per level), "
                               f"{g.nblocks - g.nleaves} parents; PPM + "
                               f"{'exact Riemann (Newton 1e-12)' if spec[head][1] == abi.RS_EXACT else 'HLLC'}, "
                               "CFL 0.8, one dt for all levels, "
                               "fine/coarse flux correction, graph-replayed step",
                   "zones_per_gpu": zones, "leaf_blocks": g.nleaves,
                   "l2": f"inputs larger than L2 (state {g.nblocks * 256 * 40 / 1e6:.0f} MB plus guard buffers "
                         f"{g.nleaves * 576 * 40 / 1e6:.0f} MB)", "path": head, "hierarchy_build_s": build_s},
        "paths": {n: {"value": zones / (ms[n] * 1e-3), "ms_per_step": ms[n], "launches_per_step": launches[n],
                      **({f"rel_l1_vs_{ref_of[n]}": errs[n][0], f"rel_linf_vs_{ref_of[n]}": errs[n][1],
                          f"rel_l1_momentum_vector_vs_{ref_of[n]}": errs[n][2]} if n in errs else {}),
                      **({"launch_shape": tunings[n]} if n in tunings else {})} for n in ms},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "peak_kind": peak_kind,
                     "kernel": "one AMR step (restriction, halos, k_sig, per-level k_dir), 80 B/leaf zone algorithmic"},
        "clocks": clocks, "gpu_launches": launches[head] * steps,
    }
    if "fp64" in ms and head != "fp64":
        line["speedup_vs_fp64"] = ms["fp64"] / ms[head]
    if e2e_ms is not None:
        line["e2e"] = {"value": zones / (e2e_ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": 6 * 8 * g.nblocks * 256,
                       "d2h_bytes_per_step": 10 * 8 * g.nblocks * 256, "ms_per_step": e2e_ms,
                       "path": "flash_hy_upload + flash_hy_step + flash_hy_compute_dt + flash_hy_download, "
                               "every node's FLASH UNK (11 vars), pinned host memory; the upload packs DENS, VEL*, "
                               "EINT, ENER and the download the 10 owned variables"}
    if cpu_r is not None:
        line["cpu_baseline"] = cpu_r
    if regrid_info is not None:
        line["refinement_cycle"] = regrid_info
    if training is not None:
        line["training"] = training
    torch.cuda.empty_cache()
    return line


def amr_summary(line):
    p = line["paths"]
    out = {"workload": line["config"]["workload"], "zones": line["config"]["zones_per_gpu"],
           "path": line["config"]["path"], "value": line["value"], "unit": UNIT,
           "ms_per_step": {n: round(v["ms_per_step"], 4) for n, v in p.items()},
           "launches_per_step": {n: v["launches_per_step"] for n, v in p.items()},
           "errors": {n: {k: v[k] for k in v if k.startswith("rel_")} for n, v in p.items()
                      if any(k.startswith("rel_") for k in v)}}
    if "fp64" in p:
        out["speedup_vs_fp64"] = {n: p["fp64"]["ms_per_step"] / v["ms_per_step"] for n, v in p.items()}
    if "fp64_exact" in p:
        out["speedup_vs_fp64_exact"] = {n: p["fp64_exact"]["ms_per_step"] / v["ms_per_step"] for n, v in p.items()}
    if "training" in line:
        out["training_hydro_face_states"] = line["training"]["hydro_face_states"]
    return out


def riemann_summary(line):
    p = line["paths"]
    return {"workload": line["config"]["workload"], "unit": "solves/s",
            "solves_per_s": {n: v["solves_per_s"] for n, v in p.items()},
            "mean_newton_evaluations": {n: v["mean_iters"] for n, v in p.items()},
            "fallback_frac_learned": p["learned"]["fallback_frac"],
            "consulted_frac": line["consulted_frac"],
            "mean_newton_evaluations_where_consulted": {n: v["mean_iters_where_consulted"] for n, v in p.items()},
            "network_dense_ms": line["network_dense_ms"],
            "roofline": line["roofline"],
            "speedup_learned_vs_two_rarefaction": line["speedup_vs_two_rarefaction"],
            "max_rel_pstar_diff_learned_vs_tr": line["max_rel_pstar_diff_learned_vs_tr"]}


# ---------------------------------------------------------------------------
# main
# ---------------------------------------------------------------------------
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nblk", type=int, default=64, help="blocks per axis (64 -> 512^3)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-extra", action="store_true", help="KH workload: skip the AMR and isolated-Riemann keys")
    ap.add_argument("--no-tune", action="store_true", help="keep the default launch shapes (no autotuning)")
    ap.add_argument("--sweep", choices=["xyz", "zyx"], default=None,
                    help="sweep order of the mixed paths before any tuning (the autotuner may change it)")
    ap.add_argument("--no-regrid", action="store_true", help="AMR workload: skip the refinement-cycle timing")
    ap.add_argument("--nspecies", type=int, default=0, help="KH workload: species advected with the flow")
    ap.add_argument("--nmass-scalars", type=int, default=0, help="KH workload: mass scalars advected with the flow")
    ap.add_argument("--workload", default="kh", choices=["kh", "riemann", "amr"])
    ap.add_argument("--amr-nblk", type=int, default=32, help="root blocks per axis of the AMR hierarchy")
    ap.add_argument("--riemann-n", type=int, default=100_000_000)
    # training set of the isolated workload's network (smaller for profiling runs)
    ap.add_argument("--riemann-train-n", type=int, default=2_000_000)
    ap.add_argument("--riemann-epochs", type=int, default=8)
    ap.add_argument("--paths", default="fp64,fp64_exact,mixed,mixed_exact,mixed_learned",
                    help="comma list of paths to time; profiling runs use one")
    args = ap.parse_args()
    paths = args.paths.split(",")
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    warmup = max(3, args.warmup)
    args.warmup = warmup
    if args.workload == "amr" and args.impl == "ours":
        if rank != 0:
            return 0
        print(json.dumps(amr_run(args, paths, e2e=not args.no_e2e, regrid=not args.no_regrid,
                                 cpu=not args.no_cpu)))
        return 0
    if args.workload == "riemann" and args.impl == "ours":
        if rank != 0:
            return 0
        print(json.dumps(riemann_run(args)))
        return 0

    if args.impl == "reference":
        if rank != 0:
            return 0
        r = cpu_sample(args.nblk, steps=args.steps, warmup=warmup)
        line = {"metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
                "warmup": warmup, "ms_per_step": r["ms_per_step_median"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded KH noise)",
                "config": kh_config(args, world=args.gpus), "impl": "reference", "cpu_baseline": r,
                "e2e": {"value": r["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return 0

    import torch
    dist = None
    if world > 1:
        import torch.distributed as tdist
        import datetime
        torch.cuda.set_device(local)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = tdist
    else:
        torch.cuda.set_device(0)
    dev = local if world > 1 else 0

    from flash5_b200.hydro import Hydro
    g, unk, abi = kh_workload(args.nblk, nguard=0, nspecies=args.nspecies, nmass_scalars=args.nmass_scalars)
    zones = g.ncells
    peak, peak_kind = measured_peaks()
    if world > 1:
        # weak scaling: N copies of the KH box stacked along z, one per rank
        # (periodic), sharded by blocks with a ghost-block exchange each step
        from flash5_b200.grid import UniformGrid
        from flash5_b200.shard import ShardedHydro, ShardPlan
        gg = UniformGrid(3, (8, 8, 8), (args.nblk, args.nblk, args.nblk * world), hi=(1.0, 1.0, float(world)),
                         bc="periodic", nguard=0)
        plan = ShardPlan(gg, world, rank)
        c = gg.coords[plan.local]
        base = (c[:, 2] % args.nblk) * args.nblk * args.nblk + c[:, 1] * args.nblk + c[:, 0]
        unk_local = np.ascontiguousarray(unk[base])
        zones = len(plan.owned) * 512

    # path -> (precision, Riemann solver, learned guess, error reference path)
    spec = {"fp64": (abi.PREC_FP64, abi.RS_HLLC, 0, None),
            "fp64_fma": (abi.PREC_FP64_FMA, abi.RS_HLLC, 0, "fp64"),
            "fp64_exact": (abi.PREC_FP64, abi.RS_EXACT, 0, None),
            "mixed": (abi.PREC_MIXED, abi.RS_HLLC, 0, "fp64"),
            "mixed_exact": (abi.PREC_MIXED, abi.RS_EXACT, 0, "fp64_exact"),
            "mixed_learned": (abi.PREC_MIXED, abi.RS_EXACT, 1, "fp64_exact")}
    ms, outs, dts, launches, clocks, e2e_ms, e2e_guard, training = {}, {}, None, {}, None, None, None, None
    tunings = {}
    for name in paths:
        pr, rsv, learned, _ = spec[name]
        params = abi.default_params(gamma=5.0 / 3.0, precision=pr, riemann_solver=rsv, learned_guess=learned)
        weights = None
        if learned:
            weights, training = train_guess(g, unk, abi, dev, dts)
        if world > 1:
            h = ShardedHydro(params, gg, world, rank, device=dev, dist=dist)
            if weights is not None:
                h.h.set_guess_weights(weights)
            h.upload(unk_local)
        else:
            h = Hydro(params, g, device=dev)
            if weights is not None:
                h.set_guess_weights(weights)
            h.upload(unk)
        tuned = None
        if args.sweep and params.precision == abi.PREC_MIXED:
            hh = h.h if world > 1 else h
            hh.tuning = dict(hh.tuning, mx_sweep=abi.SWEEP_ZYX if args.sweep == "zyx" else abi.SWEEP_XYZ)
        if not args.no_tune:
            hh = h.h if world > 1 else h
            dt0 = dts[0] if dts is not None else hh.compute_dt()[0]
            best, trials = hh.autotune(dt0, steps=2)
            tuned = {"best": best, "trials_ms": {"/".join(str(v) for v in t.values()): round(m, 4)
                                                 for t, m in trials},
                     "trial_key": "sig_threads/dir_threads/mx_threads/mx_runs/mx_sweep"}
        headline = name == paths[-1]
        sampler = ClockSampler(dev) if headline else None
        ms[name], used, launches[name] = run_device(h, args.steps, warmup, dts=dts, sampler=sampler, dist=dist)
        if tuned is not None:
            tunings[name] = tuned
        if dts is None:
            dts = used            # later paths replay the first path's dt sequence
        if headline:
            clocks = sampler.summary()
        hh = h.h if world > 1 else h
        st = hh.export_state(torch)
        outs[name] = st[:, :len(plan.owned) * 512] if world > 1 else st
        if headline and not args.no_e2e and world == 1:
            pinned = torch.empty(unk.shape, dtype=torch.float64, pin_memory=True)
            host = pinned.numpy()
            host[...] = unk
            e2e_ms = run_e2e(h, host, max(3, min(args.steps, 8)), 3)
            del host, pinned
        h.close()
        if headline and not args.no_e2e and world == 1:
            e2e_guard = e2e_guard_inclusive(params, weights, dev)
    head = paths[-1]
    errs = {n: device_errors(outs[n], outs[spec[n][3]]) for n in outs if spec[n][3] in outs}
    outs.clear()
    torch.cuda.empty_cache()
    if dist is not None:
        for n in ms:
            ms[n] = dist_max(dist, ms[n])
        if e2e_ms is not None:
            e2e_ms = dist_max(dist, e2e_ms)
    total = gg.ncells if world > 1 else zones
    value = total / (ms[head] * 1e-3)
    if rank == 0:
        extra = {}
        if world == 1 and not args.no_extra:
            extra["amr"] = amr_summary(amr_run(args, ["fp64", "fp64_exact", "mixed", "mixed_exact", "mixed_learned"],
                                               e2e=False, regrid=False, cpu=False))
            extra["riemann"] = riemann_summary(riemann_run(args))
        cpu = None if (args.no_cpu or world > 1) else cpu_sample(args.nblk)
        achieved = zones * BYTES_PER_ZONE / (ms[head] * 1e-3) / 1e9
        notes = {"fp64": "plain FP64 HLLC, no FMA contraction; bit-identical to the CPU oracle in the tests",
                 "fp64_fma": "FP64 HLLC with FMA contraction",
                 "fp64_exact": "FP64, exact Riemann solver (two-rarefaction start, Newton to 1e-12); the FP64 "
                               "reference of the exact-solver paths, matches the CPU oracle to 1e-10 in the tests",
                 "mixed": "FP32 reconstruction, FP64 HLLC and update",
                 "mixed_exact": "FP32 reconstruction, FP64 exact Riemann (two-rarefaction start) and update",
                 "mixed_learned": "FP32 reconstruction, FP64 exact Riemann started from the BF16 tensor-core MLP "
                                  "guess (trained on this run's harvested face states), FP64 update"}
        fl = FLOPS_PER_ZONE.get(head)
        compute = None
        if fl is not None:
            zps = zones / (ms[head] * 1e-3)
            compute = {"flops_per_zone": {"f64": fl["f64"], "f32": fl["f32"]},
                       "f64_tflops": zps * fl["f64"] / 1e12, "f32_tflops": zps * fl["f32"] / 1e12,
                       "f64_peak_tflops": FP64_PEAK_TFLOPS, "f32_peak_tflops": FP32_PEAK_TFLOPS,
                       "f64_frac": zps * fl["f64"] / 1e12 / FP64_PEAK_TFLOPS,
                       "f32_frac": zps * fl["f32"] / 1e12 / FP32_PEAK_TFLOPS, "peak_kind": "nominal",
                       "fp64_pipe_pct_ncu": fl["fp64_pipe_pct"],
                       "note": "FLOPs per zone-update counted by ncu (SASS dadd/dmul/dfma, fadd/fmul/ffma; FMA = "
                               "2) on the 160^3 step; peaks = 148 SMs x 64 FP64 / 128 FP32 FMA lanes x 2 x "
                               "1965 MHz"}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": warmup,
            "ms_per_step": ms[head], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 reconstruction, f64 Riemann/update" + (", bf16 MLP guess" if head == "mixed_learned" else "")
                     if head.startswith("mixed") else "f64",
            "data": "synthetic (seeded KH noise)",
            "config": kh_config(args, world=world,
                                riemann="exact (Newton 1e-12)" if spec[head][1] == abi.RS_EXACT else "HLLC",
                                head=head),
            "paths": {n: {"value": total / (ms[n] * 1e-3), "ms_per_step": ms[n], "note": notes[n],
                          **({f"rel_l1_vs_{spec[n][3]}": errs[n][0], f"rel_linf_vs_{spec[n][3]}": errs[n][1],
                              f"rel_l1_momentum_vector_vs_{spec[n][3]}": errs[n][2]} if n in errs else {}),
                          **({"launch_shape": tunings[n]} if n in tunings else {})} for n in ms},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": TRAFFIC_PER_ZONE[head] * zones if head in TRAFFIC_PER_ZONE else None,
                         "traffic_note": "DRAM bytes per step (per GPU), ncu at 160^3 scaled by zones",
                         "peak_kind": peak_kind,
                         "kernel": "one hydro step (k_sig + k_dir x,y,z), 80 B/zone algorithmic",
                         **({"compute": compute} if compute else {})},
            "clocks": clocks,
            "gpu_launches": launches[head] * args.steps,
            **extra,
        }
        if training is not None:
            line["training"] = training
        if "fp64" in ms and head != "fp64":
            line["speedup_vs_fp64"] = ms["fp64"] / ms[head]
        if e2e_ms is not None:
            nsp = args.nspecies + args.nmass_scalars
            line["e2e"] = {"value": total / (e2e_ms * 1e-3), "unit": UNIT,
                           "h2d_bytes_per_step": (6 + nsp) * 8 * zones, "d2h_bytes_per_step": (5 + nsp) * 8 * zones,
                           "ms_per_step": e2e_ms,
                           "path": "flash_hy_upload + flash_hy_step + flash_hy_compute_dt + flash_hy_download, "
                                   "interior-only FLASH UNK (11 vars), pinned host memory; the upload packs DENS, "
                                   "VEL*, EINT, ENER, the download the 5 state variables, from which the host "
                                   "writes the 10 owned ones (PRES, TEMP, GAMC, GAME, ENER by the gamma law; host "
                                   "threads gather / scatter, copies pipelined by sub-chunk)"}
            if e2e_guard is not None:
                line["e2e_guard_inclusive"] = e2e_guard
        if cpu is not None:
            line["cpu_baseline"] = cpu
        print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
