"""Throughput of the PM step on B200: particle-steps/s at 512^3 particles /
512^3 mesh, FP32 (and the same run in FP64 on the GPU), against the
reference's own CPU code on the host cores.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--mbits 9] [--f 1] [--no-fp64]

A step is one leapfrog step of the solver (drift, CIC deposit, Poisson solve,
gather + kick) over all particles. The workload is the 3D throughput box:
N = 2^mbits particles per side on an (f N)^3 mesh, L = 500 Mpc/h, scale-free
P(k) ~ k^-1.5 (sigma 0.83 at 8 Mpc/h, seeded Philox white noise), Zel'dovich
start at a = 0.05 and da = 0.0475 (20 steps reach a = 1). Particle state
(3.2 GB at 512^3 in FP32) and meshes are far larger than L2, so no L2 flush is
needed between steps.

Multi-GPU: the PM step does not shard (one box per GPU); N > 1 runs N
independent replicas (seed + rank) with no data-path collective, timed as the
max over ranks ("scaling": "weak").

Output: one JSON line on rank 0 (see the keys below).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

L_BOX, NS, A0, DA = 500.0, -1.5, 0.05, 0.0475
METRIC = "PM particle-steps/s at 512^3 (FP32 vs FP64 GPU at P(k) err<1e-3); adjoint/fwd time"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--mbits", type=int, default=9)
    ap.add_argument("--f", type=int, default=1)
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--no-cic", action="store_true")
    ap.add_argument("--no-fof", action="store_true")
    ap.add_argument("--no-mesh2", action="store_true")
    ap.add_argument("--no-tune", action="store_true", help="skip the autotuner (its trial launches), e.g. for a launch list")
    return ap.parse_args()


def workload_name(mbits, f):
    n = 1 << mbits
    return f"pm3d_{n}^3_particles_{f * n}^3_mesh_L{int(L_BOX)}_ns{NS}"


# ------------------------------------------------------------------ clocks --
class Clocks:
    """Samples the SM clock and the clock-event (throttle) reasons while the
    timed region runs: NVML read-only queries every 10 ms from a thread, or
    nvidia-smi every 200 ms when NVML is unavailable."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index):
        self.index = index
        self.p = None
        self.samples = []  # (sm_mhz, max_mhz, set of reasons)
        self.thread = None

    def _nvml_sample(self):
        nv, h = self.nv, self.h
        bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
        try:
            sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
            r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
            self.samples.append((float(sm), float(self.mx), {n for n, b in bits.items() if r & b}))
        except Exception:
            pass

    def _nvml_loop(self):
        import time as _t
        while not self.stop:
            self._nvml_sample()
            _t.sleep(0.01)

    def __enter__(self):
        self.stop = False
        try:
            import threading
            import pynvml as nv
            nv.nvmlInit()
            self.nv, self.h = nv, nv.nvmlDeviceGetHandleByIndex(self.index)
            self.mx = nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM)
            self.thread = threading.Thread(target=self._nvml_loop, daemon=True)
            self.thread.start()
            return self
        except Exception:
            self.thread = None
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *a):
        self.stop = True
        self.smi_once = False
        if self.thread is not None:
            self.thread.join(timeout=2)
            if not self.samples:  # a region shorter than the thread's start-up: one reading at its end
                self._nvml_sample()
            if not self.samples:  # NVML answered nothing: one nvidia-smi reading at the end
                try:
                    r = subprocess.run(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                        "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=20)
                    self._parse_smi(r.stdout)
                    self.smi_once = True
                except (OSError, subprocess.TimeoutExpired):
                    pass
        if self.p:
            self.p.terminate()
            try:
                out, _ = self.p.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()
                out, _ = self.p.communicate()
            self._parse_smi(out)

    def _parse_smi(self, out):
        for l in out.splitlines():
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                self.samples.append((float(f[1]), float(f[2]),
                                     {n for n, v in zip(self.NAMES, f[5:9]) if v.lower().startswith("active")}))
            except ValueError:
                continue

    def summary(self):
        sm = [x[0] for x in self.samples]
        mx = self.samples[-1][1] if self.samples else None
        reasons = set().union(*[x[2] for x in self.samples]) if self.samples else set()
        source = "nvml 10 ms" if self.thread is not None else "nvidia-smi 200 ms"
        if getattr(self, "smi_once", False):
            source = "nvidia-smi once at the end (nvml gave no reading)"
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm), "source": source}


def clocks_disturbed(c):
    """True for a clock record that rejects a timing: a hardware or thermal
    slowdown, or a median SM clock below 90% of the maximum with no reason
    active. The power cap alone (sw_power_cap) is normal and kept."""
    if set(c.get("reasons", [])) & {"hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown"}:
        return True
    sm, mx = c.get("sm_mhz"), c.get("sm_max_mhz")
    return bool(sm and mx and not c.get("reasons") and sm < 0.9 * mx)


# ------------------------------------------------------------ distributed --
def dist_init(n):
    if n <= 1:
        return 0, 1, None
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    rank = int(os.environ.get("RANK", 0))
    local = int(os.environ.get("LOCAL_RANK", rank))
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    return rank, dist.get_world_size(), dist


def barrier(dist):
    if dist is not None:
        dist.barrier()


def max_over_ranks(x, dist, device="cuda"):
    """Max of x over all ranks (device "cpu" for the gloo backend)."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ------------------------------------------------------------------- fof --
def fof_bench(cb, Xh, n, dev, steps, reps=3):
    """The `fof` tool's groups (b = 0.2 linking length) on the final 512^3
    snapshot: device positions to device tags (conan_fof_run_device, CUDA
    events, inputs resident in HBM), and end to end through conan_fof_run with
    host buffers. Size-independent checks: the same tags on every run, and the
    numbering of the groups in order of their lowest particle index."""
    import torch
    Np = n ** 3
    ll = 0.2 * L_BOX / n
    eng = cb.FoF(3, Np, L_BOX, ll, device=dev)
    xd = torch.from_numpy(Xh).to(f"cuda:{dev}")
    td = torch.empty(Np, dtype=torch.int64, device=f"cuda:{dev}")
    s = torch.cuda.current_stream(dev)
    ng = eng.run_device(xd.data_ptr(), td.data_ptr(), s.cuda_stream)  # warm-up
    first = td.clone()
    ms = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        ng = eng.run_device(xd.data_ptr(), td.data_ptr(), s.cuda_stream)
        e1.record(s)
        torch.cuda.synchronize(dev)
        ms.append(e0.elapsed_time(e1))
    cm = torch.cummax(td, 0)[0]
    numbering_ok = bool(td[0].item() == 1 and torch.equal(td, first) and cm[-1].item() == ng and
                        bool(((cm[1:] - cm[:-1]) <= 1).all().item()) and bool((td <= cm).all().item()))
    mass = torch.bincount(td - 1)
    big = int((mass >= 10).sum().item())
    largest = int(mass.max().item())
    del xd, td, first, cm, mass
    eng(Xh)  # warm-up of the host path
    t0 = time.perf_counter()
    tags_h, _ = eng(Xh)
    e2e_s = time.perf_counter() - t0
    eng.close()
    return {"workload": f"final {n}^3 FP32 snapshot ({steps} steps from a={A0}, da={DA}), b=0.2: linking length 0.2 L/N",
            "linking_length": ll, "ms": min(ms), "particles_per_s": Np / (min(ms) * 1e-3),
            "groups": ng, "groups_ge_10": big, "largest_group": largest, "checks_ok": numbering_ok,
            "e2e": {"particles_per_s": Np / e2e_s, "seconds": e2e_s, "h2d_bytes": Xh.nbytes,
                    "d2h_bytes": tags_h.nbytes, "what": "conan_fof_run: host positions in, host tags out"}}


def fof_tool_vs_reference(cb, n_sample=128, max_seconds=60.0):
    """The whole `fof` tool (snapshot file in, text file out) on a 128^3 box
    with the throughput box's spacing (L = 125 Mpc/h) run to a = 1 on the GPU:
    the reference's binary (oracle/_ref/conan_ref, single-threaded kd-tree)
    against this build's `conan fof`, same file and options; the two text
    outputs must agree after the header and history."""
    import tempfile
    import numpy as np
    from conan_b200.conanfile import ConanFile
    mb = int(math.log2(n_sample))
    L = L_BOX * n_sample / 512
    H = {"dim": 3, "mbits": mb, "size": L, "ns": NS, "smooth": 0, "scale-free": 1, "scale": 8.0, "sigma": 0.83,
         "seed": 5}
    phi = cb.compute_potential(H, cb.generate_random_field(H, precision="fp64"), precision="fp64")
    g = cb.Gravity(3, n_sample, 1, L, precision="fp32")
    g.run(phi, A0, DA, 20)
    X, P = g.state()
    g.close()
    ref = ROOT / "oracle" / "_ref" / "conan_ref"
    out = {"sample": f"{n_sample}^3 particles, L={L}, 20 steps a=0.05->1, b=0.2"}
    with tempfile.TemporaryDirectory() as w:
        c = ConanFile(header={"L": repr(L), "N": str(n_sample), "dim": "3"})
        c.update_history("bench snapshot")
        c.add("pos", X)
        c.add("mom", P)
        c.write(f"{w}/s.conan")
        args = ["fof", "-f", f"{w}/s.conan", "-l", repr(0.2 * L / n_sample)]
        t0 = time.perf_counter()
        subprocess.run([str(ROOT / "conan_b200" / "bin" / "conan"), *args, "-i", "gpu"], cwd=w, check=True,
                       capture_output=True)
        out["gpu_tool_s"] = time.perf_counter() - t0
        if ref.exists():
            t0 = time.perf_counter()
            r = subprocess.run([str(ref), *args, "-i", "ref"], cwd=w, capture_output=True,
                               timeout=max_seconds * 10)
            out["reference_tool_s"] = time.perf_counter() - t0
            if r.returncode == 0:
                body = [open(f"{w}/{k}.fof.10000.txt").read().split("\n# history\n", 1)[1].split("\n\n", 1)[1]
                        for k in ("gpu", "ref")]
                out["outputs_identical"] = body[0] == body[1]
            out["reference_cores"] = 1
    return out


# ------------------------------------------------------------- reference --
def _reference_lib():
    """The reference's own code compiled from its sources (oracle/_ref), or None."""
    import ctypes
    reflib = ROOT / "oracle" / "_ref" / "libconan_ref.so"
    if not reflib.exists():
        return None
    R = ctypes.CDLL(str(reflib))
    R.ref_time_threads.restype = ctypes.c_double
    R.ref_max_threads.restype = ctypes.c_int
    return R


def _reference_potential(mbits, L, seed=3):
    """The box's potential on the CPU from the reference's mt19937 white noise
    (CPU restatement of _generate_random_field and _compute_potential,
    src/ic/ic.cc:37-117); not timed."""
    from oracle import cpu as oracle
    noise = oracle.noise_mt19937(seed, (1 << mbits) ** 3)
    return oracle.potential(3, mbits, L, oracle.grf_scale_free(3, mbits, L, NS, False, 8.0, 0.83, noise))


def cpu_reference(mbits=9, threads=(0, 1)):
    """Times the reference's own PM step, Gravity<3>::drift + kick
    (src/run/nbody.hh:97-133, compiled from its sources into oracle/_ref), on
    one box of 2^mbits particles and cells per side with the throughput box's
    cell size (L = 500 Mpc/h at 512^3), spectrum and time step: one solver
    state, one step per entry of `threads` (0: all host threads, the
    reference's OpenMP default; 1: a single thread, on which its
    `omp critical` deposit runs faster). Without oracle/_ref, one step of the
    CPU restatement."""
    import ctypes
    n = 1 << mbits
    L = L_BOX * n / 512
    phi = _reference_potential(mbits, L)
    R = _reference_lib()
    per = {}
    if R is not None:
        allthreads = R.ref_max_threads()
        th = (ctypes.c_int * len(threads))(*threads)
        sec = (ctypes.c_double * len(threads))()
        t_init = R.ref_time_threads(3, n, 1, ctypes.c_double(L), ctypes.c_double(68.5), ctypes.c_double(1.0),
                                    ctypes.c_double(0.0), phi.ctypes.data_as(ctypes.c_void_p), ctypes.c_double(A0),
                                    ctypes.c_double(DA), len(threads), th, sec)
        for t, x in zip(threads, sec):
            per[allthreads if t == 0 else t] = x
        kind = "reference"
    else:
        from oracle import cpu as oracle
        X, P = oracle.zeldovich(3, n, L, phi, A0, A0 + DA / 2)
        t0 = time.perf_counter()
        oracle.drift(3, n, 68.5, 1.0, 0.0, X, P, A0, DA)
        oracle.kick(3, n, 1, L, 68.5, 1.0, 0.0, X, P, A0 + DA / 2, DA)
        per[os.cpu_count()] = time.perf_counter() - t0
        t_init, kind = None, "port"
    best = min(per, key=per.get)
    what = "reference FP64 CPU code" if kind == "reference" else "CPU restatement of the reference (FP64)"
    return {"value": n ** 3 / per[best], "unit": "particle-steps/s", "cores": best, "kind": kind,
            "sample": f"one leapfrog step (drift + kick) of a {n}^3-particle/{n}^3-mesh box, L={L:g} Mpc/h, "
                      f"ns={NS}, from a={A0}, per thread count; {what}; value = the faster thread count",
            "seconds_per_step_by_threads": {str(k): v for k, v in sorted(per.items())},
            "init_seconds": t_init, "steps": 1, "seconds": per[best]}


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", 0))
    if rank != 0:
        return
    # One reference step of the full box takes minutes on the host cores, so
    # a step here is one leapfrog step of the same box (all threads, then one
    # thread, on one solver state); the warm-up steps have no counterpart (no
    # JIT or caches to warm).
    r = cpu_reference(mbits=args.mbits)
    line = {"metric": METRIC, "value": r["value"], "unit": "particle-steps/s", "n_gpus": args.gpus,
            "steps": r["steps"], "warmup": args.warmup, "ms_per_step": 1e3 * r["seconds"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded mt19937 white noise, scale-free GRF)", "impl": "reference",
            "config": {"workload": workload_name(args.mbits, args.f), "sample": r["sample"]},
            "cpu_baseline": {"value": r["value"], "unit": r["unit"], "cores": r["cores"], "kind": r["kind"],
                             "sample": r["sample"], "seconds_per_step_by_threads": r["seconds_per_step_by_threads"]},
            "e2e": {"value": r["value"], "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def oracle_parity(cb, dev):
    """FP32 GPU runs against the FP64 CPU oracle (the reference's algorithm)
    on the same white noise, as checks beside the CPU baseline:
    the 3D 128^3 box (L = 100, n_s = -2 smoothed at one cell, 50 steps from
    a = 0.02) and the 32^3 class of the 96-box ensemble (32 boxes, 40 steps)."""
    import numpy as np
    from oracle import cpu as oracle
    out = {}
    N, mb, L = 128, 7, 100.0
    noise = oracle.noise_mt19937(2, N ** 3)
    phi = oracle.potential(3, mb, L, oracle.grf_scale_free(3, mb, L, -2.0, True, 0.78125, 0.83, noise))
    Xr, _ = oracle.run(3, N, 1, L, 68.5, 1.0, 0.0, phi, 0.02, 0.0196, 50)
    _, Pkr, cr = oracle.power_spectrum(3, N, L, oracle.md_cic(3, N, L, Xr) - 1.0)
    g = cb.Gravity(3, N, 1, L, precision="fp32", device=dev)
    g.run(phi, 0.02, 0.0196, 50)
    X, _ = g.state()
    _, Pk, _ = g.power_spectrum(len(cr))
    g.close()
    d = (X - Xr) / (L / N)
    d = (d + N / 2) % N - N / 2
    m = (cr > 0) & (np.arange(len(cr)) > 0)
    out["c2_3d_128_fp32_vs_oracle"] = {
        "position_rms_cells": float(np.sqrt(np.mean(d ** 2))), "position_max_cells": float(np.abs(d).max()),
        "pk_ratio_max_abs_dev": float(np.max(np.abs(Pk[m] / Pkr[m] - 1))), "shells": int(m.sum()),
        "what": "ic -d 3 -b 7 -L 100 --scale-free -n -2 --smooth --scale 0.78125 --seed 2; run -a0 0.02 "
                "-da 0.0196 -n 50; FP32 GPU vs FP64 CPU oracle, same mt19937 noise and potential"}
    from conan_b200.ensemble import Ensemble, standard_members
    members = standard_members()[:32]
    e = Ensemble(members, precision="fp32", device=dev)
    e.init()
    e.run()
    gp = np.array([e.power_spectrum(i, 17)[1] for i in range(32)])
    e.close()
    rp = []
    for mb5, Lm, ns, seed in members:
        nz = cb.white_noise({"dim": 3, "mbits": mb5, "seed": seed}, device=dev)
        ph = oracle.potential(3, mb5, Lm, oracle.grf_scale_free(3, mb5, Lm, ns, False, 8.0, 0.83, nz))
        Xm, _ = oracle.run(3, 1 << mb5, 1, Lm, 68.5, 1.0, 0.0, ph, 0.05, 0.95 / 40, 40)
        rp.append(oracle.power_spectrum(3, 1 << mb5, Lm, oracle.md_cic(3, 1 << mb5, Lm, Xm) - 1.0, 17)[1])
    rp = np.array(rp)
    out["c5_ensemble_32_class_fp32_vs_oracle"] = {
        "mean_pk_max_rel_err": float(np.max(np.abs(gp.mean(0)[1:] / rp.mean(0)[1:] - 1))),
        "worst_member_pk_max_rel_err": float(np.max(np.abs(gp[:, 1:] / rp[:, 1:] - 1))),
        "what": "32 boxes of 32^3 (ns from default_rng(6), seeds 1000+i), 40 steps a=0.05->1, batched FP32 run "
                "vs FP64 CPU oracle on the same white noise"}
    return out


# ------------------------------------------------------------------- ours --
def algorithmic_bytes(kernel, Np, Nc, fp64):
    """Bytes a kernel must move by definition (FP32; x2 for FP64):
    deposit 12 Np + 4 Nc (positions in, density out); gather+kick+drift
    48 Np + 4 Nc (positions and momenta in and out, potential in); the fused
    gather+kick+drift+deposit kernel does the work of both except writing the
    density, which its accumulator conversion does: 60 Np + 4 Nc."""
    s = 2 if fp64 else 1
    if kernel.endswith("_deposit"):
        return s * (60 * Np + 4 * Nc)
    if kernel.startswith("gather_kick"):
        return s * (48 * Np + 4 * Nc)
    if kernel == "deposit":
        return s * (12 * Np + 4 * Nc)
    return None


def dram_traffic(kernel, workload):
    """DRAM bytes per launch of `kernel` on `workload` from the committed ncu
    summary (profiles/dram_traffic.txt), or None when it holds no such line."""
    try:
        for line in open(ROOT / "profiles" / "dram_traffic.txt"):
            if line.startswith("#"):
                continue
            kv = dict(x.split("=", 1) for x in line.split() if "=" in x)
            if kv.get("kernel") == kernel and kv.get("workload") == workload:
                return float(kv["traffic_bytes"])
    except OSError:
        pass
    return None


def fd_check(dev, eps_list=(1e-3, 1e-4, 1e-5), nvox=64):
    """Central finite differences of the differentiable 128^3 box's loss
    (mean squared difference of the final density to that of seed 1004, 32
    steps a = 0.05 -> 1, checkpoint 8) on 64 voxels of the white noise
    (numpy default_rng(5)), FP64 forward, against the FP64 adjoint: relative
    error per voxel, median / 90th percentile / max for each step eps."""
    import numpy as np
    import torch
    import conan_b200 as cb
    from conan_b200.autograd import DiffPM
    m = DiffPM(dim=3, mbits=7, L_box=100.0, ns=-2.0, a0=0.05, da=0.95 / 32, n=32, checkpoint_every=8,
               precision="fp64", device=dev)
    w = torch.tensor(cb.white_noise({"dim": 3, "mbits": 7, "seed": 4}, device=dev), device=f"cuda:{dev}")
    wt = torch.tensor(cb.white_noise({"dim": 3, "mbits": 7, "seed": 1004}, device=dev), device=f"cuda:{dev}")
    out = torch.empty(m.ncells, dtype=torch.float64, device=f"cuda:{dev}")
    m.forward_raw(wt, out)
    target = out.clone()

    def loss(x):
        m.forward_raw(x, out)
        return float(((out - target) ** 2).mean())

    loss(w)
    g = torch.empty_like(w)
    m.backward_raw((2 * (out - target) / m.ncells).contiguous(), g)
    g = g.cpu().numpy()
    idx = np.random.default_rng(5).choice(w.numel(), nvox, replace=False)
    res = {}
    for eps in eps_list:
        rel = []
        for i in idx:
            wp, wm = w.clone(), w.clone()
            wp[i] += eps
            wm[i] -= eps
            fd = (loss(wp) - loss(wm)) / (2 * eps)
            rel.append(abs(g[i] - fd) / max(abs(fd), 1e-30))
        rel = np.array(rel)
        res[f"{eps:g}"] = {"median_rel_err": float(np.median(rel)), "p90_rel_err": float(np.percentile(rel, 90)),
                           "max_rel_err": float(rel.max())}
    m.close()
    res["what"] = ("central FD of the loss on 64 voxels (default_rng(5)), FP64 forward, vs FP64 adjoint; "
                   "128^3 box, L=100, ns=-2, 32 steps a=0.05->1, checkpoint 8")
    return res


def run_ours(args):
    import numpy as np
    import torch
    import conan_b200 as cb

    rank, world, dist = dist_init(args.gpus)
    dev = int(os.environ.get("LOCAL_RANK", 0)) if args.gpus > 1 else 0
    torch.cuda.set_device(dev)
    mbits, f = args.mbits, args.f
    n = 1 << mbits
    Np, Nc = n ** 3, (f * n) ** 3
    H = {"dim": 3, "mbits": mbits, "size": L_BOX, "ns": NS, "smooth": 0, "scale-free": 1, "scale": 8.0,
         "sigma": 0.83, "seed": 3 + rank}
    dens = cb.generate_random_field(H, precision="fp64", device=dev)
    phi = cb.compute_potential(H, dens, precision="fp64", device=dev)
    del dens
    peaks = {}
    try:
        peaks = json.load(open(ROOT / "MEASURED_PEAKS.json"))
    except (OSError, ValueError):
        pass
    hbm = peaks.get("hbm_gbs", 6650.0)
    hbm_src = "measured" if "hbm_gbs" in peaks else "fallback"

    def timed_run(prec, profile=False, mesh_f=None):
        g = cb.Gravity(3, n, mesh_f or f, L_BOX, precision=prec, device=dev)
        s = torch.cuda.ExternalStream(g.stream_ptr())
        # warm-up: W steps from the initial conditions (plans, graphs, caches),
        # then the autotuner on that state (it puts the state back)
        g.run(phi, A0, DA, args.warmup)
        g.sync()
        tuning = g.autotune(A0 + args.warmup * DA, DA) if prec == "fp32" and not args.no_tune else None
        g.init(phi, A0, A0 + DA / 2)
        g.set_profiling(profile)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier(dist)
        torch.cuda.synchronize()
        with Clocks(dev) as clk:
            e0.record(s)
            g.run(None, A0, DA, args.steps)
            e1.record(s)
            torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        barrier(dist)
        prof = g.profile() if profile else {}
        timed_run.tuning = tuning
        return g, ms, clk.summary(), prof

    # FP32 product path (graph-captured run)
    g32, ms32, clocks, _ = timed_run("fp32")
    tuning32 = timed_run.tuning
    ms32 = max_over_ranks(ms32, dist)
    k32, P32, cnt = g32.power_spectrum()
    g32.close()
    # per-kernel profile of the same K steps (CUDA events around every launch)
    gp, msp, _, prof = timed_run("fp32", profile=True)
    # kernels only: cuFFT launches count as library work, the accumulator clear is a memset
    launches = sum(v[0] for k, v in prof.items() if not k.startswith("fft") and k != "deposit_clear")
    gp.close()
    # The headline and the profile are runs of the same K steps. A headline
    # far slower than the sum of the profiled kernels was disturbed (clocks,
    # another job on the box): it is timed once more, and both are reported.
    # The decision is taken over all ranks so that every rank runs the same
    # collectives.
    # The same holds for a run whose clock record shows a hardware or thermal
    # slowdown, or SM clocks well below their maximum with no reason given
    # (a clock lock left by someone else).
    prof_ms = sum(v[1] for v in prof.values())
    remeasured = None
    slow = prof_ms > 0 and ms32 > 1.15 * prof_ms
    if max_over_ranks(1.0 if slow or clocks_disturbed(clocks) else 0.0, dist) > 0:
        g2, ms_again, clocks_again, _ = timed_run("fp32")
        g2.close()
        remeasured = {"first_ms_per_step": ms32 / args.steps, "profile_ms_per_step": prof_ms / args.steps,
                      "first_clocks": clocks}
        ms32, clocks = max_over_ranks(ms_again, dist), clocks_again
    dom = max((k for k in prof if algorithmic_bytes(k, Np, Nc, False)), key=lambda k: prof[k][1])
    dom_ms = prof[dom][1] / prof[dom][0]
    ab = algorithmic_bytes(dom, Np, Nc, False)
    roof = {"kernel": dom, "bound": "hbm", "achieved": ab / (dom_ms * 1e-3) / 1e9, "peak": hbm,
            "unit": "GB/s", "peak_source": hbm_src, "traffic": dram_traffic(dom, workload_name(mbits, f)),
            "traffic_source": "profiles/dram_traffic.txt (ncu dram__bytes_read+write, per launch)",
            "algorithmic_bytes_per_launch": ab, "ms_per_launch": dom_ms}
    roof["frac"] = roof["achieved"] / hbm
    # the two rows the target names, each with every kernel it needs per step:
    # deposit = sort + reduce (sorted) or window deposit + accumulator
    # conversion (Lagrangian); gather = gradient mesh + gather/kick/drift
    rows = {}
    dep_b, gat_b = 12 * Np + 4 * Nc, 48 * Np + 4 * Nc
    fused = any(k.endswith("_deposit") for k in prof)
    table = ((("gather+deposit", ("fd_grad", "gather_kick_drift_deposit", "drift_deposit", "gather_kick",
                                  "deposit_mesh", "deposit_clear"), dep_b + gat_b),) if fused else
             (("deposit", ("rank", "scan", "scatter", "deposit", "deposit_mesh", "deposit_clear"), dep_b),
              ("gather", ("fd_grad", "gather_kick_drift", "gather_kick", "drift"), gat_b)))
    # with the cluster plane pass the accumulator goes straight into the
    # forward transform: no density is written, so the row does not count it
    folded = "plane_r2c" in prof
    for row, ks, ab_row in table:
        t = sum(prof[k][1] for k in ks if k in prof) / args.steps
        if folded and row in ("gather+deposit", "deposit"):
            ab_row -= 4 * Nc
        if t > 0:
            rows[row] = {"kernels": [k for k in ks if k in prof], "ms_per_step": t,
                         "algorithmic_bytes": ab_row, "achieved": ab_row / (t * 1e-3) / 1e9,
                         "frac": ab_row / (t * 1e-3) / 1e9 / hbm}
            if folded and row in ("gather+deposit", "deposit"):
                rows[row]["density"] = "converted and cleared inside plane_r2c (the forward plane transform)"

    roof["rows"] = rows
    step_bytes = 60 * Np + 24 * Nc
    kernels = {k: {"launches": v[0], "ms_total": round(v[1], 4), "share": round(v[1] / max(1e-9, sum(
        x[1] for x in prof.values())), 4)} for k, v in sorted(prof.items(), key=lambda kv: -kv[1][1])}

    # FP64 comparison path and the P(k) error of FP32 vs FP64
    fp64 = None
    if not args.no_fp64:
        g64, ms64, _, _ = timed_run("fp64")
        ms64 = max_over_ranks(ms64, dist)
        k64, P64, _ = g64.power_spectrum()
        g64.close()
        m = (cnt > 0) & (np.arange(len(cnt)) > 0)
        err = float(np.max(np.abs(P32[m] - P64[m]) / P64[m]))
        fp64 = {"value": world * Np * args.steps / (ms64 * 1e-3), "ms_per_step": ms64 / args.steps,
                "pk_max_rel_err_fp32_vs_fp64": err, "fp32_speedup": ms64 / ms32}

    # the throughput box's finer-mesh variant (2N per side: 1024^3 cells at 512^3
    # particles): FP32 and FP64 runs of the same K steps, P(k) error between them
    mesh2 = None
    if not args.no_mesh2 and f == 1:
        Nc2 = (2 * n) ** 3
        g2, ms2, _, _ = timed_run("fp32", mesh_f=2)
        ms2 = max_over_ranks(ms2, dist)
        _, P2, c2 = g2.power_spectrum()
        g2.close()
        mesh2 = {"workload": workload_name(mbits, 2), "ms_per_step": ms2 / args.steps,
                 "value": world * Np * args.steps / (ms2 * 1e-3), "unit": "particle-steps/s",
                 "step_roofline_frac": (60 * Np + 24 * Nc2) * args.steps / (ms2 * 1e-3) / 1e9 / hbm}
        if not args.no_fp64:
            g2d, ms2d, _, _ = timed_run("fp64", mesh_f=2)
            ms2d = max_over_ranks(ms2d, dist)
            _, P2d, _ = g2d.power_spectrum()
            g2d.close()
            m2 = (c2 > 0) & (np.arange(len(c2)) > 0)
            mesh2["fp64_ms_per_step"] = ms2d / args.steps
            mesh2["pk_max_rel_err_fp32_vs_fp64"] = float(np.max(np.abs(P2[m2] - P2d[m2]) / P2d[m2]))

    # the host link of this box (one pinned 1 GiB copy each way, CUDA events):
    # the end-to-end number below moves 7.5 GB across it
    link = {}
    hb = torch.empty(1 << 30, dtype=torch.uint8).pin_memory()
    db = torch.empty(1 << 30, dtype=torch.uint8, device=f"cuda:{dev}")
    for name, dst, src in (("h2d_gbs", db, hb), ("d2h_gbs", hb, db)):
        dst.copy_(src, non_blocking=True)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        dst.copy_(src, non_blocking=True)
        e1.record()
        torch.cuda.synchronize()
        link[name] = (1 << 30) / (e0.elapsed_time(e1) * 1e-3) / 1e9
    del hb, db

    # end-to-end through the C ABI with host buffers: phi in, X and P out
    ph = torch.from_numpy(phi).pin_memory().numpy()
    Xh = torch.empty((Np, 3), dtype=torch.float64).pin_memory().numpy()
    Ph = torch.empty((Np, 3), dtype=torch.float64).pin_memory().numpy()
    g = cb.Gravity(3, n, f, L_BOX, precision="fp32", device=dev)
    g.run(ph, A0, DA, args.warmup)
    if not args.no_tune:
        g.autotune(A0 + args.warmup * DA, DA)
    g.state_into(Xh, Ph)
    barrier(dist)
    torch.cuda.synchronize()
    # every call is synchronous: host timestamps between them split the total
    t0 = time.perf_counter()
    g.init(ph, A0, A0 + DA / 2)  # potential upload (1 GB FP64) + Zel'dovich start
    t1 = time.perf_counter()
    g.run(None, A0, DA, args.steps)  # the K steps (one CUDA graph)
    t2 = time.perf_counter()
    g.state_into(Xh, Ph)  # FP64 X and P to host memory (6.4 GB)
    t3 = time.perf_counter()
    e2e_s = max_over_ranks(t3 - t0, dist)
    breakdown = {"init_upload_zeldovich_s": t1 - t0, "steps_s": t2 - t1, "state_out_s": t3 - t2,
                 "link_floor_s": phi.nbytes / (link["h2d_gbs"] * 1e9) + (Xh.nbytes + Ph.nbytes) /
                 (link["d2h_gbs"] * 1e9)}
    g.close()

    # the cic tool on the final snapshot (host positions in, host density out)
    cic = None
    if rank == 0 and not args.no_cic:
        from oracle import cpu as oracle
        cic = {}
        for s in (1, 2):
            cb.cic(Xh, 3, n, L_BOX, f=1, sub_sample=s, device=dev)  # warm-up
            t0 = time.perf_counter()
            cb.cic(Xh, 3, n, L_BOX, f=1, sub_sample=s, device=dev)
            dt = time.perf_counter() - t0
            cic[f"s{s}"] = {"points_per_s": (n * s) ** 3 / dt, "seconds": dt}
        m = 6  # CPU restatement on a 64^3 sample of the same box (one thread)
        Xs = Xh.reshape(n, n, n, 3)[:: n >> m, :: n >> m, :: n >> m].reshape(-1, 3)
        t0 = time.perf_counter()
        oracle.cic(3, 1 << m, L_BOX, 1, 2, Xs)
        dt = time.perf_counter() - t0
        cic["cpu_port_s2"] = {"points_per_s": (2 << m) ** 3 / dt, "cores": 1,
                              "sample": "64^3 particles (every 8th lattice point), s=2, f=1"}
        cic["what"] = ("conan_cic on the final 512^3 FP32 snapshot, f=1 (512^3 mesh), s=1 and s=2 (1024^3 "
                       "interpolated points); host positions in, host density out")

    # the fof tool on the final snapshot, and the whole tool against the reference's
    fof = None
    if rank == 0 and not args.no_fof:
        fof = fof_bench(cb, Xh, n, dev, args.steps)
        if not args.no_cpu:
            fof["tool_128"] = fof_tool_vs_reference(cb)

    adjoint = None
    if not args.no_adjoint and rank == 0:
        from conan_b200 import autograd as ag
        adjoint = ag.benchmark_adjoint_ratio(device=dev)
        adjoint["finite_differences"] = fd_check(dev)

    ensemble = None
    if not args.no_ensemble and rank == 0:
        from conan_b200.ensemble import Ensemble
        e = Ensemble.standard(device=dev)
        e.init()
        e.run()  # warm-up: builds and instantiates the graph
        run_ms = min(e.run() for _ in range(3))
        e.forward_adjoint()
        _, adj_ms = e.last_ms()
        n_ens = e.total_particles()
        e.run()
        _, pk32 = e.mean_power_spectrum(17)
        tuning = e.describe()
        e.close()
        # the same ensemble in FP64: ensemble-mean P(k) error of the FP32 run
        e = Ensemble.standard(device=dev, precision="fp64")
        e.init()
        e.run()
        _, pk64 = e.mean_power_spectrum(17)
        m = (pk64 > 0) & (np.arange(len(pk64)) > 0)  # bin 0: the k = 0 mode, zero up to rounding
        pk_err = float(np.max(np.abs(pk32[m] - pk64[m]) / pk64[m]))
        ensemble = {"workload": "96 boxes: 32 x 32^3, 32 x 64^3, 32 x 128^3 particles = mesh, L=100, "
                                "ns in {-2.5,-2,-1.5,-1} (default_rng(6)), seeds 1000+i, 40 steps a=0.05->1, FP32",
                    "particles": n_ens, "run_ms": run_ms,
                    "particle_steps_per_s": n_ens * 40 / (run_ms * 1e-3),
                    "forward_adjoint_ms": adj_ms, "mean_pk_max_rel_err_fp32_vs_fp64": pk_err,
                    "tuning": tuning}
        e.close()

    # CPU leg (rank 0, N = 1): the reference's own step on a bounded sample of
    # the box (256^3 particles and cells with the same cell size, one step on
    # one thread: about half a minute on the host cores), and the oracle
    # parity checks of the FP32 path
    cpu, parity = None, None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_reference(mbits=min(mbits, 8), threads=(1,))
        parity = oracle_parity(cb, dev)

    if rank == 0:
        value = world * Np * args.steps / (ms32 * 1e-3)
        line = {
            "metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms32 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded Philox white noise, scale-free GRF, Zel'dovich start)",
            "config": {"workload": workload_name(mbits, f), "particles": Np, "mesh_cells": Nc, "L": L_BOX,
                       "ns": NS, "a0": A0, "da": DA, "precision": "fp32 (lattice index + fp32 displacement)",
                       "gradient": "fd4", "l2": "inputs larger than L2 (3.2 GB particle state), no flush",
                       "parallelism": f"replicas x{world}"},
            "roofline": roof,
            "step_roofline": {"achieved": step_bytes * args.steps / (ms32 * 1e-3) / 1e9, "peak": hbm,
                              "unit": "GB/s", "frac": step_bytes * args.steps / (ms32 * 1e-3) / 1e9 / hbm,
                              "algorithmic_bytes_per_step": step_bytes},
            "kernels": kernels,
            "tuning": {"state": f"after the {args.warmup} warm-up steps (a = {A0 + args.warmup * DA:g})",
                       "knobs": tuning32},
            "gpu_launches": launches,
            "fp64_gpu": fp64,
            "mesh_2n": mesh2,
            "adjoint": adjoint,
            "ensemble": ensemble,
            "cic": cic,
            "fof": fof,
            "e2e": {"value": world * Np * args.steps / e2e_s, "unit": "particle-steps/s",
                    "h2d_bytes_per_step": phi.nbytes / args.steps,
                    "d2h_bytes_per_step": (Xh.nbytes + Ph.nbytes) / args.steps,
                    "what": "conan_pm_init (potential upload, Zel'dovich start) + conan_pm_run (K steps) + "
                            "conan_pm_get_state, pinned host buffers",
                    "seconds": e2e_s, "breakdown": breakdown, "host_link": link},
            "cpu_baseline": cpu,
            "oracle_parity": parity,
            "clocks": clocks,
            "remeasured": remeasured,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference_arm(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
