"""The reference driver's time loop, restated over any object with the ``HIT`` interface.

src/MAIN.cpp:336-357 (viscosity from the Taylor-Reynolds number) and
src/MAIN.cpp:413-442 (main loop, including the QA-build per-step report line)
are restated here so that the GPU solver (``spns_b200.HIT``) and the CPU oracle
are driven by exactly the same sequence of calls.  File outputs of the loop
(src/MAIN.cpp:449-484) are not part of the time step and are left to callers.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Callable, List, Optional

from .params import HitArgs, read_forced_ek


@dataclass
class StepRecord:
    """One QA report line: ``Time, iter, Dt, Ek, Om, ReLambda`` (src/MAIN.cpp:440)."""
    time: float
    iter: int
    dt: float
    ek: float
    om: float
    relambda: float

    def qa_line(self) -> str:
        return ("Time: %f,    iter: %8d,    Dt: %e,    Ek: %e,    Om: %e,    ReLambda: %8.3f"
                % (self.time, self.iter, self.dt, self.ek, self.om, self.relambda))


def initial_viscosity(hit, args: HitArgs, forced_ek=None) -> None:
    """src/MAIN.cpp:336-357."""
    if not args.isReLambda:
        return
    if args.isForcedEk:
        Ek_tot = float(sum(forced_ek[1:args.last_input_rad + 1]))
        Om_tot = float(sum(2 * K * K * forced_ek[K] for K in range(1, args.last_input_rad + 1)))
        nu = Ek_tot / args.ReLambda * math.sqrt(20.0 / 3.0 / Om_tot)
    elif args.is_file_init:
        nu = hit.getEk_init_file() / args.ReLambda * math.sqrt(20.0 / 3.0 / hit.getEnstrophy_init_file())
    else:
        nu = 1.0e-3
    hit.setnu(nu)
    hit.Recalculate_TimeStep()


def run(hit, args: HitArgs, max_steps: Optional[int] = None, qa_report: bool = True,
        on_step: Optional[Callable[[int], None]] = None) -> List[StepRecord]:
    """Main loop of src/MAIN.cpp:413-442 until ``Final_Time`` (or ``max_steps``)."""
    forced_ek = read_forced_ek(args.EkFilename, args.last_input_rad) if args.isForcedEk else None
    initial_viscosity(hit, args, forced_ek)
    records: List[StepRecord] = []
    it = 0
    while hit.gettime() < args.Final_Time:
        if max_steps is not None and it >= max_steps:
            break
        hit.New_Fractional_Step_Method()
        if it == 0 and args.isReLambda and not args.isForcedEk and not args.is_file_init:
            hit.Forcing_Reynolds_Lambda(args.ReLambda)
            hit.Recalculate_TimeStep()
        if args.isForcedEk and hit.gettime() < args.Final_Forced_Time:
            hit.Forcing_Energy_Cascade(forced_ek, args.last_input_rad, args.isNullifyMissingEk)
        if args.isReLambda_iter and it % args.ReLambda_Freq == 0:
            hit.Forcing_Reynolds_Lambda(args.ReLambda)
            hit.Recalculate_TimeStep()
        it += 1
        if qa_report:
            hit.Recalculate_Reynolds_Lambda()
            records.append(StepRecord(hit.gettime(), it, hit.getAt(), hit.getEk_Tot(), hit.getOk_Tot(),
                                      hit.getReLambda()))
        if on_step is not None:
            on_step(it)
    return records
