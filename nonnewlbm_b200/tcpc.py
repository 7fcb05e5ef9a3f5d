"""TCPC case driver: the drop-in for the ``sim_tcpc`` process (solver/sim_tcpc/sim_tcpc.cu).

Same command line (sim_tcpc.cu:70-125), same materials and unit conversions
(sim_tcpc.cu:52-68, 787-838), same time loop and output counters (solver/lbm3d/core.h:
1473-1628, counter semantics of solver/lbm3d/state.h:65-70), same results layout
(``results_<id>/log_rank000`` and ``results_<id>/vtk3D/rank000_data_<n>.vtk``), same VTK
field set and order (sim_tcpc.cu:716-784) and exit codes (0 ok, 1 error or usage, 2 when the
boundary setup flags ``terminate``).  The step itself runs in libnnlbm.so.

    python -m nonnewlbm_b200.tcpc --geometry runtime/geometry.vtk --material gx \\
        --ivc-mls 8 --svc-mls 4.833333333 --case-id v1_gx [options]

Extra options of this build: --dtype (f32 default, f16, bf16, f64), --collision (CUM
default; KBC_N1..N4, KBC_C1..C4, MRT_LES, BGK), --cy-mode (none = the single-rank reference,
ref-fd, local-neq), --equilibrium, --bounce-back (fullway default, the reference's wall
nodes; halfway), --device, --results-root, --ramp-steps, and the state
checkpoint knobs the reference keeps in State (state.h:229-257): --wall-time SECONDS (save
the state and stop when reached) and --savestate-period SECONDS (wall-clock period of the
`savestate` flag check).  A `results_<id>/loadstate` flag resumes from the saved state
(checkpoint.py).
"""
from __future__ import annotations

import os
import sys
import time
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from . import capi, checkpoint, units, vtk
from .lattice import CaseSpec, Lattice

USAGE = ("Usage: ./sim_tcpc --geometry geometry.vtk --material newtonian|sx|gx "
         "--ivc-mls VALUE --svc-mls VALUE --case-id NAME [options]\n"
         "Options:\n"
         "  --final-time VALUE          Physical final time in seconds, default 10\n"
         "  --vtk-period VALUE          3D VTK period in seconds, default 0.1\n"
         "  --print-period VALUE        Log period in seconds, default 0.1\n"
         "  --stat-reset-period VALUE   Statistics reset period, default disabled\n"
         "  --lbm-viscosity VALUE       LBM reference viscosity, default 1e-4\n"
         "  --block-size VALUE          CUDA y-block size, default 32 (accepted; the launch shape is autotuned)\n")


@dataclass
class TcpcOptions:
    """TcpcOptions (sim_tcpc.cu:25-38) plus the options of this build."""
    geometry: str = "geometry.vtk"
    material: str = "newtonian"
    case_id: str = "tcpc_manual"
    ivc_mls: float = 8.0
    svc_mls: float = 4.833333333
    final_time: float = 10.0
    vtk_period: float = 0.1
    print_period: float = 0.1
    stat_reset_period: float = -1.0
    lbm_viscosity: float = 1.0e-4
    block_size: int = 32
    dtype: str = "f32"
    collision: str = "CUM"
    cy_mode: str = "none"
    equilibrium: str = "inv_cum_ref"
    bounce_back: str = "fullway"    # fullway (wall nodes, the reference) | halfway
    device: int = 0
    results_root: str = "."
    ramp_steps: int = 0
    wall_time: float = -1.0         # State::wallTime (state.h:256), seconds; <= 0 disables
    savestate_period: float = -1.0  # cnt[SAVESTATE].period in wall-clock seconds (core.h:1594)


def parse_args(argv) -> TcpcOptions:
    """parseArgs (sim_tcpc.cu:84-125): unknown arguments and missing values raise."""
    o = TcpcOptions()
    num = {"--ivc-mls": "ivc_mls", "--svc-mls": "svc_mls", "--final-time": "final_time", "--vtk-period": "vtk_period",
           "--print-period": "print_period", "--stat-reset-period": "stat_reset_period",
           "--lbm-viscosity": "lbm_viscosity", "--wall-time": "wall_time", "--savestate-period": "savestate_period"}
    text = {"--geometry": "geometry", "--material": "material", "--case-id": "case_id", "--output-id": "case_id",
            "--dtype": "dtype", "--collision": "collision", "--cy-mode": "cy_mode", "--equilibrium": "equilibrium",
            "--results-root": "results_root", "--bounce-back": "bounce_back"}
    ints = {"--block-size": "block_size", "--device": "device", "--ramp-steps": "ramp_steps"}
    i = 0
    while i < len(argv):
        a = argv[i]
        if a in ("--help", "-h"):
            sys.stderr.write(USAGE)
            raise SystemExit(0)
        if a in num or a in text or a in ints:
            if i + 1 >= len(argv):
                raise ValueError(f"Missing value for {a}")
            v = argv[i + 1]
            if a in num:
                setattr(o, num[a], _atof(v))
            elif a in ints:
                setattr(o, ints[a], int(float(v)) if v.strip() else 0)
            else:
                setattr(o, text[a], v)
            i += 2
        else:
            raise ValueError(f"Unknown argument '{a}'")
    return o


def _atof(s: str) -> float:
    try:
        return float(s)
    except ValueError:
        return 0.0  # std::atof returns 0 on malformed input


class Counter:
    """state.h:65-70: fires when time >= count * period and period > 0."""

    def __init__(self, period: float):
        self.period = period
        self.count = 0

    def action(self, t: float) -> bool:
        return self.period > 0 and t >= self.count * self.period


class TcpcRun:
    def __init__(self, o: TcpcOptions):
        self.o = o
        wall, (nx, ny, nz), dx = vtk.read_geometry(o.geometry)
        mat = units.material_by_name(o.material)
        conv = units.lattice_units(mat, dx, o.lbm_viscosity)
        self.mat, self.dx, self.dt = mat, dx, conv["dt"]
        self.conv = conv
        self.shape = (nx, ny, nz)
        self.dir = Path(o.results_root) / f"results_{o.case_id}"
        self.dir.mkdir(parents=True, exist_ok=True)
        self.map, self.counts, rc, self.wall_flags = capi.tcpc_labels(wall, with_wall_flags=True)
        self.terminate = rc == capi.ERR_AREA
        cy = (conv["nu0"], conv["lambda"], conv["a"], conv["n"])
        self.lat = Lattice(CaseSpec((nx, ny, nz), collision=o.collision, dtype=o.dtype, equilibrium=o.equilibrium,
                                    cy_mode=o.cy_mode if mat.carreau_yasuda else "none", nu=conv["nu"], cy=cy,
                                    bounce_back=o.bounce_back),
                           device=o.device)
        self.lat.set_map(self.map)
        self.ivc = units.flux_lbm(o.ivc_mls, dx, self.dt)
        self.svc = units.flux_lbm(o.svc_mls, dx, self.dt)
        self.lat.set_inflow(ivc_flux=self.ivc, svc_flux=self.svc)
        self.lat.init_equilibrium()
        self.iterations = 0
        self.prev_iter = 0
        c = self.counts
        self.log(f"case={o.case_id} material={mat.name} density={mat.density:e} nu_inf={mat.nu_inf:e} "
                 f"physDl={dx:e} physDt={self.dt:e}")
        self.log(f"prescribed flows: IVC={o.ivc_mls:e} ml/s SVC={o.svc_mls:e} ml/s")
        if c["left_area"] <= 0 or c["right_area"] <= 0:
            self.log(f"error: zero inlet area detected: left={c['left_area']} right={c['right_area']}")
        if c["outlet5"] <= 0 or c["outlet6"] <= 0:
            self.log(f"error: zero outlet area detected: outlet5={c['outlet5']} outlet6={c['outlet6']}")
        self.log(f"geometry labels: fluid={c['fluid']} wall={c['wall']} IVC(label3)={c['left_area']} "
                 f"SVC(label4)={c['right_area']} outlet5={c['outlet5']} outlet6={c['outlet6']}")
        self.log(f"input VTK cap-label counts before plane imposition: label3={c['vtk3']} label4={c['vtk4']} "
                 f"label5={c['vtk5']} label6={c['vtk6']}")

    # -- logging (state.hpp:53-78) -------------------------------------------------------
    def log(self, msg: str) -> None:
        stamp = time.strftime("%Y-%m-%d %H:%M:%S")
        with open(self.dir / "log_rank000", "a") as f:
            f.write(f"{stamp} {msg}\n")
        print(msg)

    def phys_time(self, it=None) -> float:
        return self.dt * (self.iterations if it is None else it)

    # -- outputs (sim_tcpc.cu:684-784) ---------------------------------------------------
    def output_fields(self):
        """The fields of StateTcpc::outputData (sim_tcpc.cu:716-784), computed on the device."""
        mat, c = self.mat, self.conv
        nu_lbm_ref = self.dt / self.dx / self.dx * mat.nu_inf
        cy = (c["nu0"], c["lambda"], c["a"], c["n"]) if mat.carreau_yasuda else None
        return self.lat.output_fields(self.dx, self.dt, mat.density, nu_lbm_ref, cy=cy,
                                      steps_summed=max(1, self.iterations - self.prev_iter), wall_flags=self.wall_flags)

    def write_vtk(self, count: int) -> Path:
        d = self.dir / "vtk3D"
        d.mkdir(parents=True, exist_ok=True)
        p = d / f"rank000_data_{count}.vtk"
        vtk.write_output(p, self.map, self.dx, self.phys_time(), count, self.output_fields())
        self.log(f"[vtk {p} written, time {self.phys_time():f}, cycle {count}] ")
        return p

    # -- the time loop (core.h:1473-1628) ------------------------------------------------
    # -- checkpoint (state.hpp:1724-1756, core.h:1511-1602) --------------------------------
    _CNT_INDEX = {"stat": checkpoint.STAT_RESET, "print": checkpoint.PRINT, "vtk": checkpoint.VTK3D,
                  "save": checkpoint.SAVESTATE}

    def save_state(self, cnt, forced: bool = False) -> bool:
        """State::saveState: with the `savestate` flag present (or forced) write the state;
        the flag is then replaced by `savestate_done`, and a forced save creates `loadstate`."""
        if not (forced or checkpoint.flag_exists(self.dir, "savestate")):
            return False
        self.log("[saveState invoked]")
        counters = {self._CNT_INDEX[k]: (c.count, c.period) for k, c in cnt.items()}
        checkpoint.save_state(self.dir, self.lat, self.iterations, self.o.final_time, counters, self.map)
        if not forced:
            checkpoint.flag_delete(self.dir, "savestate")
            checkpoint.flag_create(self.dir, "savestate_done")
        else:
            checkpoint.flag_create(self.dir, "loadstate")
        return True

    def load_state(self, cnt) -> None:
        """State::loadState: the saved populations, fields, sums, iteration and counters."""
        self.log("[loadState invoked]")
        cfg = checkpoint.load_state(self.dir, self.lat, labels=self.map)
        self.iterations = cfg["iterations"]
        self.prev_iter = self.iterations - cfg["stats_count"]
        for k, c in cnt.items():
            if self._CNT_INDEX[k] in cfg["counters"]:
                c.count = cfg["counters"][self._CNT_INDEX[k]][0]

    def run(self) -> int:
        o = self.o
        cnt = {"print": Counter(o.print_period), "stat": Counter(o.stat_reset_period), "vtk": Counter(o.vtk_period),
               "save": Counter(o.savestate_period)}
        if checkpoint.flag_exists(self.dir, "loadstate"):
            self.load_state(cnt)
        # the launch shape of the step kernel is timed on copies of the state, not taken from
        # --block-size (sim_tcpc.cu:118-119)
        self.lat.autotune(stats=True, macro=True)
        self.log(f"\nSTART: simulation LBM:{o.collision} dimensions {self.shape[0]} x {self.shape[1]} x {self.shape[2]} "
                 f"lbmVisc {self.conv['nu']:e} physDl {self.dx:e} physDt {self.dt:e}")
        t_wall0 = time.perf_counter()
        # the wall clock is checked after every call; with a checkpoint knob on, calls stay short
        max_chunk = 100 if (o.wall_time > 0 or o.savestate_period > 0) else 100000
        t1 = time.perf_counter()
        prev_mlups_it = 0
        total = int(np.prod(self.shape))
        # initial snapshot: AfterSimUpdate before the loop (core.h:1564)
        self._after(cnt)
        quit_ = False
        while not quit_:
            # steps until a counter fires or the final time passes
            k = 0
            while True:
                k += 1
                t = self.dt * (self.iterations + k)
                if (cnt["vtk"].action(t) or cnt["stat"].action(t) or cnt["print"].action(t) or t > o.final_time
                        or self.terminate or k >= max_chunk):
                    break
            if o.ramp_steps > 0:
                rows = []
                for j in range(k):
                    s = min(1.0, (self.iterations + j + 1) / o.ramp_steps)
                    rows.append([self.ivc * s, self.svc * s, s])
                self.lat.set_schedule(np.array(rows))
            self.lat.step(k, stats=True, macro=True)
            self.iterations += k
            write_info = self._after(cnt)
            if write_info and self.iterations > 1:
                t2 = time.perf_counter()
                lups = (self.iterations - prev_mlups_it) * total / max(t2 - t1, 1e-12)
                t1 = t2
                prev_mlups_it = self.iterations
                wt = time.perf_counter() - t_wall0
                eta = wt * (o.final_time - self.phys_time()) / max(self.phys_time(), 1e-30)
                self.log(f"MLUPS={lups * 1e-6:.1f} iter={self.iterations} t={self.phys_time():1.3f}s dt={self.dt:1.2e} "
                         f"lbmVisc={self.conv['nu']:1.2e} WT={wt:.0f}s ETA={eta:.0f}s")
            wall = time.perf_counter() - t_wall0
            if o.wall_time > 0 and wall >= o.wall_time:
                self.log(f"wallTime reached: {wall:.0f} / {o.wall_time:.0f} [sec]")
                self.log("maximum wall time reached")
                self.save_state(cnt, forced=True)
                quit_ = True
            elif cnt["save"].action(wall):
                self.save_state(cnt)
                cnt["save"].count += 1
            if self.phys_time() > o.final_time:
                self.log("physFinalTime reached")
                quit_ = True
            if self.terminate:
                self.log("terminate flag triggered")
                quit_ = True
        self.lat.close()
        return 2 if self.terminate else 0

    def _after(self, cnt) -> bool:
        t = self.phys_time()
        write_info = False
        if cnt["vtk"].action(t):
            self.write_vtk(cnt["vtk"].count)
            cnt["vtk"].count += 1
            write_info = True
        if cnt["print"].action(t):
            write_info = True
            cnt["print"].count += 1
        if cnt["stat"].action(t):
            self.lat.stat_reset()
            self.prev_iter = self.iterations
            cnt["stat"].count += 1
        return write_info


def main(argv=None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    try:
        o = parse_args(argv)
        return TcpcRun(o).run()
    except SystemExit:
        raise
    except Exception as e:  # sim_tcpc.cu:852-856
        sys.stderr.write(f"sim_tcpc: {e}\n")
        sys.stderr.write(USAGE)
        return 1


if __name__ == "__main__":
    raise SystemExit(main())
