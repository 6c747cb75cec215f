"""Benchmark: time steps per second of the forced 512^3 DNS (FFT grid 768^3) on B200.

Workload (the forced-DNS configuration): N=512 retained modes per axis (3/2-rule
FFT grid 768^3), seeded solenoidal field with E(k) ~ k^4 exp(-2 (k/4)^2) and
u_rms=1, constant-power forcing eps=0.1 on shells K=1..2 (the reference's
disabled forcing block src/HIT_LES.cpp:243-278 with eps_in=0.1), nu=4.90e-4
(k_max*eta = 1.5 with k_max=N/2), self-adaptive time step (kappa scheme) with
C_At=0.5, FP64 plain form.  A "step" is one HIT::New_Fractional_Step_Method.

--gpus N runs N independent replicas (one box per GPU, one process per GPU);
the solver has no data-path collective, so `value` is the sum over ranks
(N*K steps / max over ranks of the device time) and scaling is weak.

--impl reference times the reference solver on the host cores (oracle/_ref:
src/*.cpp of adalbal/SpNS compiled unchanged against single-process MPI and
FFTW stand-ins, the oracle's OpenMP FFT in place of FFTW's threads; where it
was not built, the CPU oracle, a C restatement of the same solver) on a bounded
sample of the same workload, and prints the same JSON line with
"impl": "reference".
"""
from __future__ import annotations

import argparse
import json
import math
import os
import re
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_BOX = 512
KP = 4.0
EPS = 0.1
C_AT = 0.5
SEED = 2024
METRIC = "time steps/s, forced DNS N=512 (FFT 768^3), FP64"
# kernels behind the per-pass event names at N=512, FP64 (the z pass at length 768 is the
# persistent pair-staged kernel)
KERNEL_SYMBOL = {"k3_z": "k3_rot_staged<double,768,E=12,1 pencil per block,2 slots in shared memory>", "k1_inv_x": "k1_inv_x<double,768,12,4>",
                 "k2_inv_y": "k2_inv_y<double,768,24,8>", "k4_fwd_y": "k4_fwd_y<double,768,24,8>",
                 "k5_fwd_x": "k5_fwd_x<double,768,24,4>", "k6_sweep": "k6_sweep<double,kappa>"}


def nu_for(N: int, eps: float = EPS) -> float:
    """nu with k_max*eta = 1.5, eta=(nu^3/eps)^(1/4), k_max=N/2."""
    kmax = N / 2
    eta = 1.5 / kmax
    return (eta ** 4 * eps) ** (1.0 / 3.0)


def box_args(N: int, self_adaptive: bool = True, nxy: int = 0, shape=None):
    """Box of the forced DNS; `nxy` or `shape` (Nx, Ny, Nz) give reduced boxes for profiling."""
    from spns_b200.params import HitArgs
    Nx, Ny, Nz = shape or (nxy or N, nxy or N, N)
    M = lambda n: (3 * n) // 2  # noqa: E731
    return HitArgs(Nx=Nx, Ny=Ny, Nz=Nz, Mx=M(Nx), My=M(Ny), Mz=M(Nz), nu=nu_for(N), C_Smag=0.0, C_At=C_AT, Lx=1, Ly=1, Lz=1,
                   omega_x=0.0, omega_y=0.0, omega_z=0.0, Nx_file=-1, Ny_file=-1, Nz_file=-1, isReLambda=False,
                   isInitialFieldFromBinaryFile=False, isInitialFieldFromASCIIFile=False, isNotCubic=False,
                   isRotating=False, isLES=False, isComplexConjugateCorrected=False, isSelfAdaptive=self_adaptive)


def algorithmic_bytes(N: int, self_adaptive: bool = True, word: int = 16, form: str = "rotational", shape=None):
    """Bytes each kernel must move once (arrays read + written, each counted once).

    S0 = compact spectral field, S1 = after the x transform, S2 = after the y
    transform (complex elements of `word` bytes).  Rotational form (default, exact
    with the edge correction): K1 3 S0 -> 6 S1 (u and the vorticity), K2 6 S1 -> 6 S2,
    K3 6 S2 -> 3 S2; advective form: 3 S0 -> 6 S1, 6 S1 -> 9 S2, 9 S2 -> 3 S2.  Then K4 3 S2 -> 3 S1,
    K5 3 S1 -> 3 S0 (nonlinear term G), K6 reads G, u, R^{n-1} (+ u^{n-1}) and writes
    R^n, u^{n+1}.  The edge correction moves O(M^2) bytes (negligible)."""
    Nx, Ny, Nz = shape or (N, N, N)
    Kx, Ky, Kz = 2 * (Nx // 2) + 1, 2 * (Ny // 2) + 1, Nz // 2 + 1
    Mx, My = (3 * Nx) // 2, (3 * Ny) // 2
    S0, S1, S2 = Ky * Kx * Kz, Ky * Mx * Kz, My * Mx * Kz
    n1, n2 = (6, 9) if form == "advective" else (6, 6)
    return {
        "k1_inv_x": (3 * S0 + n1 * S1) * word,
        "k2_inv_y": (n1 * S1 + n2 * S2) * word,
        "k3_z": (n2 * S2 + 3 * S2) * word,
        "k4_fwd_y": (3 * S2 + 3 * S1) * word,
        "k5_fwd_x": (3 * S1 + 3 * S0) * word,
        "k6_sweep": ((18 if self_adaptive else 15) * S0) * word,
    }, dict(S0=S0, S1=S1, S2=S2)


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle sampling while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = os.path.join("/tmp", f"spns_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        if self.proc is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as fh:
            for line in fh:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax = float(parts[2])
                except ValueError:
                    continue
                for nm, v in zip(names, parts[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(nm)
        sm.sort()
        med = sm[len(sm) // 2] if sm else None
        return {"sm_mhz": med, "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(n_gpus: int):
    if n_gpus <= 1 and "RANK" not in os.environ:
        return 0, 1, 0, None
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    rank, world = int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", n_gpus))
    local = int(os.environ.get("LOCAL_RANK", rank))
    torch.cuda.set_device(local)
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    return rank, world, local, dist


def reduce_max(dist, value: float) -> float:
    from spns_b200.replicas import max_over_ranks
    return max_over_ranks(value, dist, "cuda")


def barrier(dist):
    if dist is not None:
        dist.barrier()


# ---------------------------------------------------------------------------
# CPU oracle timing (reference arm and cpu_baseline)
# ---------------------------------------------------------------------------
def cpu_sample(n_sample: int, steps: int, threads: int):
    """Times `steps` oracle steps of the same workload at N=n_sample; returns s/step."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from spns_b200.fields import seeded_spectral_field
    a = box_args(n_sample)
    a.nu = nu_for(N_BOX)
    h = O.OracleHIT(a, k41_ranks=1, nthreads=threads, eps_forcing=EPS)
    h.set_compact(seeded_spectral_field(n_sample, n_sample, n_sample, kp=KP, seed=SEED))
    h.Recalculate_Velocity_Antitransform()
    h.Recalculate_TimeStep()
    h.New_Fractional_Step_Method()  # first step (untimed)
    t0 = time.perf_counter()
    for _ in range(steps):
        h.New_Fractional_Step_Method()
    return (time.perf_counter() - t0) / steps


REF_EXE = os.path.join(ROOT, "oracle", "_ref", "spns_ref")


def ref_run(workdir: str, n: int, final_time: float, threads: int):
    """One run of the compiled reference solver on an n^3 box: (wall s, steps, final time)."""
    with open(os.path.join(workdir, "params"), "w") as fh:
        fh.write(f"Nx\t{n}\nNy\t{n}\nNz\t{n}\nnu\t{nu_for(N_BOX):.6e}\nFinal_Time\t{final_time:.9e}\n"
                 f"C_At\t0.5\nSelfAdaptiveTimestep\t1\nOMP_Threads\t{threads}\n")
    t0 = time.perf_counter()
    r = subprocess.run([REF_EXE, "params"], cwd=workdir, capture_output=True, timeout=1800)
    wall = time.perf_counter() - t0
    out = r.stdout.decode(errors="replace")
    if r.returncode != 0:
        raise RuntimeError(f"reference solver failed ({r.returncode}): {out[-500:]}")
    steps = int(re.search(r"Final time-steps:\s*(\d+)", out).group(1))
    t_end = float(re.search(r"Final time:\s*(\S+)", out).group(1))
    return wall, steps, t_end


def ref_sample(n_sample: int, steps: int, threads: int):
    """Seconds per step of the compiled reference solver at N=n_sample: a one-step run and a
    run of about 1 + `steps` steps, both timed whole; their difference cancels the set-up
    (K41 field, allocation, planning).  Returns (s/step, steps timed)."""
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        w1, n1, dt1 = ref_run(d, n_sample, 1e-12, threads)
        w2, n2, _ = ref_run(d, n_sample, dt1 * (steps + 1.5), threads)
    if n2 <= n1:
        raise RuntimeError("reference sample ran no extra step")
    return (w2 - w1) / (n2 - n1), n2 - n1


def cpu_step_seconds(n_sample: int, steps: int, threads: int):
    """(s/step, kind, description) of the CPU reference at N=n_sample: the compiled
    reference solver where it was built, else the oracle port."""
    if os.path.exists(REF_EXE):
        s, k = ref_sample(n_sample, steps, threads)
        return s, "reference", (f"the reference solver (src/*.cpp compiled unchanged; MPI/FFTW stand-ins, the oracle's "
                                f"OpenMP FFT in place of FFTW) at N={n_sample}, {k} steps timed, {s:.3f} s/step; "
                                f"unforced (its eps-forcing block is disabled), K41 initial field, same nu and kappa scheme")
    s = cpu_sample(n_sample, steps, threads)
    return s, "port", f"{steps} steps of the CPU oracle (C restatement) at N={n_sample}, {s:.3f} s/step"


def fft_work(N: int) -> float:
    M = (3 * N) // 2
    return M ** 3 * math.log2(M ** 3)


def cpu_baseline_block(threads: int, n_sample: int = 96, steps: int = 3):
    s, kind, desc = cpu_step_seconds(n_sample, steps, threads)
    scale = fft_work(N_BOX) / fft_work(n_sample)
    v = 1.0 / (s * scale)
    return {"value": v, "unit": "steps/s", "cores": threads, "kind": kind,
            "sample": (f"{desc} (FFT {(3 * n_sample) // 2}^3), extrapolated to N={N_BOX} by FFT work "
                       f"M^3 log2 M^3 (x{scale:.1f}); the reference layout needs ~200 GB of host RAM at N={N_BOX}")}


def _timed_steps(h, n: int) -> float:
    """Wall seconds of n steps through the public API (graph replays, synchronised)."""
    t0 = time.perf_counter()
    h.New_Fractional_Step_Method(n)
    return time.perf_counter() - t0


def fp32_accuracy_block(a, local: int, rank: int, steps: int):
    """FP32 compensated form against the FP64 form over `steps` steps of the benchmark box
    from the same seeded state: E(K) per shell, total energy and dissipation nu*Omega
    (Omega = sum of 2 k^2 E, the enstrophy integral of src/HIT_LES.cpp:490-495, 998-1002,
    so that nu*Omega = 2 nu sum k^2 E(k)).  Each form runs alone."""
    import numpy as np
    from spns_b200.hit import HIT, SPNS_FP64, SPNS_FP32_HILO
    from spns_b200.fields import seeded_spectral_field
    res = {}
    for prec in (SPNS_FP64, SPNS_FP32_HILO):
        h = HIT(a, device=local, eps_forcing=EPS, precision=prec)
        U0 = seeded_spectral_field(a.Nx, a.Ny, a.Nz, kp=KP, seed=SEED + rank)
        h.set_compact(U0)
        del U0
        h.Recalculate_Velocity_Antitransform()
        h.Recalculate_TimeStep()
        h.New_Fractional_Step_Method(steps)
        ek = h.Recalculate_Energy_Cascade()
        om = h.Recalculate_Enstrophy()
        res[prec] = (ek, float(np.sum(ek)), h.getnu() * om, h.gettime())
        h.close()
    e64, E64, d64, t64 = res[SPNS_FP64]
    e32, E32, d32, t32 = res[SPNS_FP32_HILO]
    m = e64 > 1e-6 * e64.max()
    return {"steps": steps,
            "ek_max_shell_rel_err": float(np.max(np.abs(e32[m] - e64[m]) / e64[m])),
            "energy_rel_err": abs(E32 - E64) / E64,
            "dissipation_rel_err": abs(d32 - d64) / d64,
            "time_rel_err": abs(t32 - t64) / t64,
            "fp64_energy": E64, "fp64_dissipation": d64,
            "tolerance_ek_shell": 1e-5,
            "shells_compared": "shells holding more than 1e-6 of the peak shell energy"}


def stretch_block(local: int, n: int = 1024, steps: int = 5):
    """The 1024^3 stretch of the forced DNS (FFT 1536^3) in the compensated FP32 form, which
    fits one B200 (about 162 GB; the FP64 form needs about 272 GB and runs as slabs over
    several GPUs).  Same workload as the headline box at N=1024."""
    from spns_b200.hit import HIT, SPNS_FP32_HILO, SpnsError, estimate_device_bytes
    import torch
    a = box_args(n)
    a.nu = nu_for(n)
    out = {"N": n, "fft_grid": (3 * n) // 2, "precision": "FP32 compensated form",
           "device_bytes": estimate_device_bytes(a, precision=SPNS_FP32_HILO, eps_forcing=EPS)}
    try:
        h = HIT(a, device=local, eps_forcing=EPS, precision=SPNS_FP32_HILO, k41_ranks=-1)
    except SpnsError as e:
        out["unavailable"] = str(e)
        return out
    h.seed_field(SEED, KP, 1.0)
    h.New_Fractional_Step_Method(3)
    stream = torch.cuda.ExternalStream(h.stream_handle(), device=torch.device("cuda", local))
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    h._ck(h._L.spns_step(h._h, steps))
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    energy = h.Recalculate_Energy()
    s = h.scalars()
    h.close()
    out.update({"steps": steps, "ms_per_step": ms, "steps_per_s": 1e3 / ms, "energy": energy,
                "finite": math.isfinite(s.At) and math.isfinite(energy)})
    return out


def same_n_block(local: int, n: int, threads: int, cpu_steps: int = 3, gpu_steps: int = 50):
    """The oracle and the GPU on the SAME forced-DNS box at a size the host can hold
    (N=n retained modes, FFT (3n/2)^3): measured steps/s of both, no extrapolation."""
    from spns_b200.hit import HIT
    from spns_b200.fields import seeded_spectral_field
    import torch
    s_cpu, kind, desc = cpu_step_seconds(n, cpu_steps, threads)
    a = box_args(n)
    a.nu = nu_for(N_BOX)
    h = HIT(a, device=local, eps_forcing=EPS)
    h.set_compact(seeded_spectral_field(n, n, n, kp=KP, seed=SEED))
    h.Recalculate_Velocity_Antitransform()
    h.Recalculate_TimeStep()
    h.New_Fractional_Step_Method(3)
    stream = torch.cuda.ExternalStream(h.stream_handle(), device=torch.device("cuda", local))
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    h._ck(h._L.spns_step(h._h, gpu_steps))
    e1.record(stream)
    torch.cuda.synchronize()
    gpu_s = e0.elapsed_time(e1) / 1e3 / gpu_steps
    t0 = time.perf_counter()
    for _ in range(gpu_steps):
        h.New_Fractional_Step_Method()
        h.Recalculate_Energy_Cascade()
    e2e_s = (time.perf_counter() - t0) / gpu_steps
    h.close()
    return {"N": n, "fft_grid": (3 * n) // 2, "cores": threads, "kind": kind, "cpu_sample": desc,
            "cpu_steps": cpu_steps, "cpu_steps_per_s": 1.0 / s_cpu,
            "gpu_steps": gpu_steps, "gpu_steps_per_s": 1.0 / gpu_s, "gpu_e2e_steps_per_s": 1.0 / e2e_s,
            "gpu_over_cpu": s_cpu / gpu_s, "gpu_e2e_over_cpu": s_cpu / e2e_s,
            "workload": f"the benchmark's forced DNS (same nu, eps, kappa scheme) at N={n}"}


def ensemble_block(local: int, n_boxes: int = 64, steps: int = 500, seed: int = 7):
    """64 LES boxes of uneven size advanced together (one CUDA graph per step, FP32 form,
    launch shapes per box class picked by the autotuner).

    Grids uniform in {32,48,64,96}^3 (FFT 48..144), Cs uniform in [0.10, 0.20],
    nu=1e-4, per-instance Philox seeds with k_p=3, u_rms=1, CFL dt (C_At=0.5).
    The sequential baselines step each box alone (its own CUDA graph per step),
    in the same FP32 form and in the plain FP64 form, timed over `probe` steps
    and scaled to `steps`."""
    import numpy as np
    from spns_b200.hit import HIT, Ensemble, SPNS_FP64, SPNS_FP32_HILO
    from spns_b200.serving import box_args as sbox
    rng = np.random.default_rng(seed)
    specs = [(int(rng.choice([32, 48, 64, 96])), float(rng.uniform(0.10, 0.20)), int(rng.integers(0, 2 ** 63)))
             for _ in range(n_boxes)]
    members, shapes = [], {}
    for N, cs, sd in specs:
        h = HIT(sbox(N, nu=1e-4, C_Smag=cs), precision=SPNS_FP32_HILO, device=local, k41_ranks=-1)
        h.seed_field(sd, 3.0, 1.0)
        shapes[str(N)] = h.autotune(steps=3)      # timed once per box class, then cached
        members.append(h)
    ens = Ensemble(members)
    ens.step(3)                                   # first step uncaptured, then graph capture
    t0 = time.perf_counter()
    ens.step(steps)
    t_ens = time.perf_counter() - t0
    ens.close()
    for h in members:
        h.close()
    probe = 20
    seq = {}
    for prec, name in ((SPNS_FP32_HILO, "fp32_hilo"), (SPNS_FP64, "fp64")):
        tot = 0.0
        for N, cs, sd in specs:
            h = HIT(sbox(N, nu=1e-4, C_Smag=cs), precision=prec, device=local, k41_ranks=-1)
            h.seed_field(sd, 3.0, 1.0)
            h.New_Fractional_Step_Method(3)
            tot += _timed_steps(h, probe) / probe * steps
            h.close()
        seq[name] = tot
    box_steps = n_boxes * steps
    return {"boxes": n_boxes, "steps_each": steps, "dtype": "FP32 compensated form",
            "grids": {str(N): sum(1 for s_ in specs if s_[0] == N) for N in (32, 48, 64, 96)},
            "box_steps_per_s": box_steps / t_ens, "wall_s": t_ens,
            "sequential_fp32_box_steps_per_s": box_steps / seq["fp32_hilo"],
            "sequential_plain_fp64_box_steps_per_s": box_steps / seq["fp64"],
            "speedup_vs_sequential_fp32": seq["fp32_hilo"] / t_ens,
            "speedup_vs_sequential_plain_fp64": seq["fp64"] / t_ens,
            "autotuned_shapes": {k: {"K1..K5 alternate (E=6)": v} for k, v in sorted(shapes.items(), key=lambda kv: int(kv[0]))},
            "how": "one CUDA graph per step with every box's step as a parallel branch; launch shapes per box "
                   "class picked by spns_autotune (the sequential FP32 baseline uses the same tuned shapes, the "
                   f"plain FP64 one the defaults); sequential baselines timed over {probe} steps per box and "
                   f"scaled to {steps}"}


def les_config_block(local: int, steps: int = 2000):
    """The LES configuration: rotating Smagorinsky LES (C_s=0.17, Omega=(0,0,1), nu=1e-4)
    on the non-cubic box Nx=Ny=128, Nz=256 with Lz=2 (FFT grid 192 x 192 x 384), seeded
    k_p=3 field with u_rms=1, CFL time step, `steps` steps in the compensated FP32 form
    and in the FP64 form; E(K), total energy and eddy-viscosity statistics of FP32
    against FP64 at the end."""
    import numpy as np
    from spns_b200.hit import HIT, SPNS_FP64, SPNS_FP32_HILO
    from spns_b200.params import HitArgs
    ex = lambda n, f: n * f  # noqa: E731  (even sizes)
    a = HitArgs(Nx=128, Ny=128, Nz=ex(128, 2), Mx=192, My=192, Mz=ex(192, 2), nu=1e-4, C_Smag=0.17, C_At=C_AT,
                Lx=1, Ly=1, Lz=2, omega_x=0.0, omega_y=0.0, omega_z=1.0, Nx_file=-1, Ny_file=-1, Nz_file=-1,
                isReLambda=False, isInitialFieldFromBinaryFile=False, isInitialFieldFromASCIIFile=False,
                isNotCubic=True, isRotating=True, isLES=True, isComplexConjugateCorrected=False, isSelfAdaptive=False)
    runs, rate, probe = {}, {}, 50
    for prec in (SPNS_FP64, SPNS_FP32_HILO):
        h = HIT(a, precision=prec, device=local, k41_ranks=-1)
        h.seed_field(3, 3.0, 1.0)
        h.New_Fractional_Step_Method(3)
        rate[prec] = probe / _timed_steps(h, probe)
        h.New_Fractional_Step_Method(steps - 3 - probe)
        runs[prec] = h
    e64, e32 = runs[SPNS_FP64].Recalculate_Energy_Cascade(), runs[SPNS_FP32_HILO].Recalculate_Energy_Cascade()
    m = e64 > 1e-6 * e64.max()
    n64, n32 = runs[SPNS_FP64].eddy_viscosity_stats(), runs[SPNS_FP32_HILO].eddy_viscosity_stats()
    rel = np.abs(n32 - n64) / n64
    out = {"workload": "LES C_s=0.17, Omega=(0,0,1), Nx=Ny=128, Nz=256 (Lz=2; FFT 192x192x384), nu=1e-4, "
                       f"seeded k_p=3, CFL dt, {steps} steps",
           "fp32_hilo_steps_per_s": rate[SPNS_FP32_HILO], "fp64_steps_per_s": rate[SPNS_FP64],
           "speedup_fp32_vs_fp64": rate[SPNS_FP32_HILO] / rate[SPNS_FP64],
           "ek_max_shell_rel_err": float(np.max(np.abs(e32[m] - e64[m]) / e64[m])),
           "etot_rel_err": float(abs(e32.sum() - e64.sum()) / e64.sum()),
           "nu_t_fp64_mean_rms_max": n64.tolist(), "nu_t_rel_err_mean_rms_max": rel.tolist(),
           "tolerances": {"ek_shell": 2e-5, "etot": 1e-6, "nu_t_mean_rms": 1e-6, "nu_t_max": 5e-5}}
    for h in runs.values():
        h.close()
    return out


def serving_block(local: int, n_requests: int = 40, rate: float = 20.0, seed: int = 11, budget_gb: float = 150.0):
    """Served workload: Poisson arrivals of LES/DNS runs, continuous batching.

    Grids {32,64,128,256}^3 with weights 0.4/0.3/0.2/0.1, steps uniform in
    [200, 2000], LES (Cs in [0.10, 0.20], nu in [1e-4, 1e-3]) or DNS (nu in
    [1e-3, 1e-2]) with equal odds, seeded k_p=3 spectra, FP32 form, 150 GB HBM
    budget.  The sequential plain-path baseline runs the same requests one at
    a time in FP64: each (grid, LES/DNS) class is timed alone over `probe`
    steps and the per-request times are summed."""
    from spns_b200.hit import HIT, SPNS_FP64
    from spns_b200.serving import GpuBackend, Server, summarize, synthetic_workload
    reqs = synthetic_workload(n_requests, rate=rate, seed=seed)
    srv = Server(GpuBackend(device=local), budget_bytes=int(budget_gb * 1e9), chunk=25)
    t0 = time.perf_counter()
    res = srv.run(reqs)
    makespan = time.perf_counter() - t0
    out = summarize(res, makespan)
    probe = 20
    per_step = {}
    for r in reqs:
        key = (r.args.Nx, r.args.isLES)
        if key in per_step:
            continue
        h = HIT(r.args, precision=SPNS_FP64, device=local, k41_ranks=-1)
        h.seed_field(r.seed, r.kp, r.urms)
        h.New_Fractional_Step_Method(3)
        per_step[key] = _timed_steps(h, probe) / probe
        h.close()
    seq = sum(per_step[(r.args.Nx, r.args.isLES)] * r.nsteps for r in reqs if res[r.rid].status == "done")
    out.update({
        "workload": f"{n_requests} requests, Poisson {rate:g}/s, grids 32/64/128/256 (0.4/0.3/0.2/0.1), "
                    "steps U[200,2000], LES or DNS, FP32 form, 150 GB budget",
        "peak_budget_used_gb": srv.peak_used / 1e9,
        "sequential_plain_fp64_solves_per_s": out["done"] / seq if seq > 0 else None,
        "speedup_vs_sequential_plain_fp64": (out["solves_per_s"] * seq / out["done"]) if out["done"] else None,
        "how": "latency = completion - arrival (wall clock); sequential plain path = the same requests one at a "
               f"time in FP64, per-class step time from {probe} timed steps",
    })
    return out


def run_reference(args):
    rank = int(os.environ.get("RANK", 0))
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    n_sample = args.ref_sample_n
    if os.path.exists(REF_EXE):
        # W warm-up steps inside the first (set-up cancelling) run pair, then K timed steps
        if args.warmup > 0:
            ref_sample(n_sample, args.warmup, threads)
        s, kind, desc = cpu_step_seconds(n_sample, max(1, args.steps), threads)
    else:
        for _ in range(args.warmup):
            cpu_sample(n_sample, 1, threads)
        per = [cpu_sample(n_sample, 1, threads) for _ in range(max(1, args.steps))]
        s, kind = sum(per) / len(per), "port"
        desc = f"one CPU-oracle step at N={n_sample} per timed step, {s:.3f} s/step"
    scale = fft_work(N_BOX) / fft_work(n_sample)
    value = 1.0 / (s * scale)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / value, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"forced DNS N={N_BOX} (FFT 768^3), eps=0.1 on K=1..2, self-adaptive dt",
                   "sample": f"N={n_sample} per step, extrapolated"},
        "cpu_baseline": {"value": value, "unit": "steps/s", "cores": threads, "kind": kind,
                         "sample": f"{desc}; x{scale:.1f} FFT work to N={N_BOX}"},
        "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def run_gpu(args):
    import numpy as np
    import torch
    rank, world, local, dist = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    from spns_b200.hit import HIT
    from spns_b200.fields import seeded_spectral_field
    from spns_b200.replicas import whole_job_rate

    N = args.n
    shape = tuple(int(v) for v in args.shape.split(",")) if args.shape else None
    a = box_args(N, nxy=args.nxy, shape=shape)
    h = HIT(a, device=local, eps_forcing=EPS)
    U0 = seeded_spectral_field(a.Nx, a.Ny, a.Nz, kp=KP, seed=SEED + rank)
    h.set_compact(U0)
    del U0
    h.Recalculate_Velocity_Antitransform()
    h.Recalculate_TimeStep()
    stream = torch.cuda.ExternalStream(h.stream_handle(), device=torch.device("cuda", local))

    for _ in range(args.warmup):
        h.New_Fractional_Step_Method()
    nk = h.kernels_per_step()

    # --- timed region: K steps (CUDA-graph replays) timed with events on the solver's stream ---
    barrier(dist)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record(stream)
        h._ck(h._L.spns_step(h._h, args.steps))
        ev1.record(stream)
        torch.cuda.synchronize()
    barrier(dist)
    ms = ev0.elapsed_time(ev1)
    ms_max = reduce_max(dist, ms)
    ek64 = h.Recalculate_Energy_Cascade()       # spectrum after W + K steps (FP32 comparison below)

    # --- per-kernel breakdown: the same K steps again, uncaptured, with an event before every kernel ---
    h.profile_begin(args.steps)
    h._ck(h._L.spns_step(h._h, args.steps))
    names, per = h.profile_read(args.steps)

    # --- e2e: the public API loop with a device->host read of the step's result ---
    torch.cuda.synchronize()
    barrier(dist)
    nbins = h.getlast_rad_max() + 1
    t0 = time.perf_counter()
    for _ in range(args.steps):
        h.New_Fractional_Step_Method()
        h.Recalculate_Energy_Cascade()
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    e2e_max = reduce_max(dist, e2e_s)
    s = h.scalars()
    finite = math.isfinite(s.Ek_Tot) and math.isfinite(s.At)
    h.close()

    # --- compensated FP32 form on the same initial state: same W + K steps, timed the same way ---
    fp32 = None
    if not args.no_fp32:
        from spns_b200.hit import SPNS_FP32_HILO
        h32 = HIT(a, device=local, eps_forcing=EPS, precision=SPNS_FP32_HILO)
        U0 = seeded_spectral_field(a.Nx, a.Ny, a.Nz, kp=KP, seed=SEED + rank)
        h32.set_compact(U0)
        del U0
        h32.Recalculate_Velocity_Antitransform()
        h32.Recalculate_TimeStep()
        s32 = torch.cuda.ExternalStream(h32.stream_handle(), device=torch.device("cuda", local))
        for _ in range(args.warmup):
            h32.New_Fractional_Step_Method()
        barrier(dist)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s32)
        h32._ck(h32._L.spns_step(h32._h, args.steps))
        e1.record(s32)
        torch.cuda.synchronize()
        barrier(dist)
        ms32_max = reduce_max(dist, e0.elapsed_time(e1))
        ek32 = h32.Recalculate_Energy_Cascade()
        h32.close()
        mask = ek64 > 1e-6 * ek64.max()
        fp32 = {"value": whole_job_rate(world, args.steps, ms32_max / 1e3), "unit": "steps/s",
                "ms_per_step": ms32_max / args.steps, "speedup_vs_fp64": ms_max / ms32_max,
                "dtype": "f32 transforms and products, f32 hi+lo state (~48 bits), f64 reductions/CFL/forcing",
                "ek_max_shell_rel_err_vs_fp64": float(np.max(np.abs(ek32[mask] - ek64[mask]) / ek64[mask])),
                "ek_max_abs_err_over_ek_tot": float(np.max(np.abs(ek32 - ek64)) / ek64.sum()),
                "steps_compared": args.warmup + args.steps,
                "shells_compared": "shells holding more than 1e-6 of the peak shell energy"}
        if args.accuracy_steps > 0:
            fp32["accuracy"] = fp32_accuracy_block(a, local, rank, args.accuracy_steps)

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return 0
    value = whole_job_rate(world, args.steps, ms_max / 1e3)
    e2e_value = whole_job_rate(world, args.steps, e2e_max)
    # roofline of the dominant kernel
    bytes_per, sizes = algorithmic_bytes(N, shape=(a.Nx, a.Ny, a.Nz))
    mean_ms = per.mean(axis=0)
    share = {n: float(m) for n, m in zip(names, mean_ms)}
    dom = max((n for n in names if n in bytes_per), key=lambda n: share[n])
    achieved = bytes_per[dom] / (share[dom] / 1e3) / 1e9
    peak, peak_kind = measured_peaks()
    traffic = None
    tp = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tp):
        with open(tp) as fh:
            traffic = json.load(fh).get(dom)
    step_bytes = sum(bytes_per.values())
    line = {
        "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64",
        "data": "synthetic: seeded solenoidal field, E(k)~k^4 exp(-2(k/4)^2), u_rms=1",
        "config": {"workload": f"forced DNS N={N} (FFT {(3 * N) // 2}^3), eps=0.1 on K=1..2, nu={a.nu:.3e}, "
                               "self-adaptive dt C_At=0.5, FP64 plain form",
                   "N": N, "fft_grid": (3 * N) // 2, "parallelism": f"replicas x{world}",
                   "l2": f"inputs larger than L2 (state {3 * sizes['S0'] * 16 / 1e9:.1f} GB, work buffers "
                         f"{(6 * sizes['S1'] + 9 * sizes['S2']) * 16 / 1e9:.1f} GB)",
                   "nonlinear_form": "rotational + exact +-N/2 aliasing correction (= the reference's u.grad u after projection)",
                   "finite": finite},
        "clocks": clk.summary(),
        "e2e": {"value": e2e_value, "unit": "steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 8 * nbins + 8,
                "loop": "HIT.New_Fractional_Step_Method() + Recalculate_Energy_Cascade() (E(K) to host) per step",
                "why_no_h2d": "a step takes no host input: the state stays resident on the device between steps, "
                              "as HIT keeps its fields in its own arrays in the reference's loop "
                              "(src/MAIN.cpp:413-485); the initial state is uploaded once before the loop"},
        "gpu_launches": nk * args.steps,
        "kernel_ms": share,
        "kernel_ms_note": "per-kernel CUDA-event times of K further uncaptured steps on the solver stream",
        "graphs": "timed steps replay one CUDA graph per step",
        "step_algorithmic_bytes": step_bytes,
        "step_achieved_GBps": step_bytes / (ms_max / args.steps / 1e3) / 1e9,
        "roofline": {"bound": "hbm", "kernel": dom, "kernel_symbol": KERNEL_SYMBOL.get(dom, dom),
                     "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind, "traffic": traffic,
                     "algorithmic_bytes": bytes_per[dom]},
    }
    if not args.no_les:
        line["les_config"] = les_config_block(local)
    if not args.no_ensemble:
        line["ensemble"] = ensemble_block(local)
    if not args.no_serving:
        line["serving"] = serving_block(local, n_requests=args.serving_requests)
    if not args.no_stretch:
        line["stretch_n1024_fp32"] = stretch_block(local)
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_block(os.cpu_count() or 1)
        if args.same_n:
            line["cpu_baseline"]["measured_same_n"] = same_n_block(local, args.same_n, os.cpu_count() or 1)
    # last: the driver keeps the tail of a long line
    line["fp32_hilo"] = fp32
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["spns", "reference"], default="spns")
    ap.add_argument("--n", type=int, default=N_BOX, help="retained modes per axis (default 512)")
    ap.add_argument("--shape", default="",
                    help="Nx,Ny,Nz of a reduced box for profiling one pass at its full FFT length "
                         "(e.g. 64,512,64 runs the y passes at length 768)")
    ap.add_argument("--nxy", type=int, default=0,
                    help="retained modes along x and y (default: as --n); a small value gives a reduced box "
                         "that runs the same z-pass kernel, for profiling")
    ap.add_argument("--ref-sample-n", type=int, default=96)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp32", action="store_true", help="skip the compensated FP32 form's extra line field")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the 64-box LES ensemble field")
    ap.add_argument("--no-serving", action="store_true", help="skip the served-workload field")
    ap.add_argument("--no-les", action="store_true", help="skip the LES-configuration field (FP32 vs FP64)")
    ap.add_argument("--serving-requests", type=int, default=40)
    ap.add_argument("--no-stretch", action="store_true", help="skip the 1024^3 FP32 stretch field")
    ap.add_argument("--accuracy-steps", type=int, default=100,
                    help="steps of the FP32-vs-FP64 accuracy comparison (0 skips it)")
    ap.add_argument("--same-n", type=int, default=128,
                    help="box size at which the oracle and the GPU are both measured (0 skips it)")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        return run_reference(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
