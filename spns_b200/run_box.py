"""Run one seeded box for a number of steps and report its step rate.

    python -m spns_b200.run_box --shape 64,64,512 --precision fp32 --steps 5

The box is the forced-DNS workload of bench.py (seeded k^4 exp(-2(k/4)^2)
field, u_rms=1, constant-power forcing eps=0.1 on K=1..2, kappa-scheme time
step, nu from k_max*eta = 1.5 for the largest axis) at any retained-mode shape,
in either precision and nonlinear form.  It is the small driver the kernel
profiles are taken with (a reduced box runs the same pass kernels at the full
FFT length along one axis), and a quick way to time a configuration.
"""
from __future__ import annotations

import argparse
import json
import time

from .fields import seeded_spectral_field
from .hit import HIT, SPNS_FP32_HILO, SPNS_FP64
from .params import HitArgs


def box_args(shape, nu: float, les: float = 0.0, self_adaptive: bool = True) -> HitArgs:
    Nx, Ny, Nz = shape
    M = lambda n: (3 * n) // 2  # noqa: E731
    return HitArgs(Nx=Nx, Ny=Ny, Nz=Nz, Mx=M(Nx), My=M(Ny), Mz=M(Nz), nu=nu, C_Smag=les, C_At=0.5, Lx=1, Ly=1, Lz=1,
                   omega_x=0.0, omega_y=0.0, omega_z=0.0, Nx_file=-1, Ny_file=-1, Nz_file=-1, isReLambda=False,
                   isInitialFieldFromBinaryFile=False, isInitialFieldFromASCIIFile=False, isNotCubic=False,
                   isRotating=False, isLES=les > 0, isComplexConjugateCorrected=False, isSelfAdaptive=self_adaptive)


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--shape", default="512,512,512", help="retained modes Nx,Ny,Nz (FFT grid 3N/2 per axis)")
    ap.add_argument("--precision", choices=["fp64", "fp32"], default="fp64")
    ap.add_argument("--form", choices=["rotational", "advective"], default="rotational")
    ap.add_argument("--les", type=float, default=0.0, help="Smagorinsky constant (0: DNS)")
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--eps", type=float, default=0.1)
    ap.add_argument("--seed", type=int, default=2024)
    args = ap.parse_args(argv)
    shape = tuple(int(v) for v in args.shape.split(","))
    kmax = max(shape) / 2
    nu = ((1.5 / kmax) ** 4 * args.eps) ** (1.0 / 3.0)
    prec = SPNS_FP64 if args.precision == "fp64" else SPNS_FP32_HILO
    h = HIT(box_args(shape, nu, args.les), precision=prec, eps_forcing=args.eps,
            nonlinear_form=0 if args.form == "rotational" else 2)
    h.set_compact(seeded_spectral_field(*shape, kp=4.0, seed=args.seed))
    h.Recalculate_Velocity_Antitransform()
    h.Recalculate_TimeStep()
    h.New_Fractional_Step_Method(args.warmup)
    t0 = time.perf_counter()
    h.New_Fractional_Step_Method(args.steps)
    wall = time.perf_counter() - t0
    h.profile_begin(args.steps)
    h.New_Fractional_Step_Method(args.steps)
    names, per = h.profile_read(args.steps)
    mean = per.mean(axis=0)
    out = {"shape": shape, "precision": args.precision, "form": args.form, "les": args.les, "steps": args.steps,
           "steps_per_s": args.steps / wall, "kernel_ms": {n: round(float(m), 4) for n, m in zip(names, mean)},
           "energy": h.Recalculate_Energy(), "dt": h.getAt()}
    h.close()
    print(json.dumps(out), flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
