"""Launch-shape autotuner for an Engine.

Candidates, each kept only if it is faster:
  * threads per particle of the cell-group and whole-box force kernels;
  * cells per block of the whole-box kernels (the partition of the force and
    list grids over a batch), when it has whole-box systems;
  * threads per particle x block size of the per-particle kernel (boxes with
    fewer than 3 cells per side that are too large for the whole-box kernels).
No candidate changes a result beyond FP64 rounding: the sums are
deterministic, and only the threads per particle change the order in which a
particle's pairs are summed.

mode "forces" times the force stage alone (acg_time_stage, forces only: the
trajectory is not changed); mode "step" times whole steps (acg_bench_steps:
forces, list rebuilds, kick/drift and events as they come, so the engine
advances `step_reps` steps per candidate).
"""
from __future__ import annotations

from .engine import Engine
from .init import box_length

GROUP_TPP = (1, 2, 4)
BOX_CELLS = (1, 2, 4, 8)
SMALL_SHAPES = ((1, 64), (1, 128), (2, 128), (2, 256), (4, 128), (4, 256), (8, 256))


def _kind(e: Engine, r: int) -> str:
    """Which kernels serve system r: whole-box (2 to 4 cells per side, N <=
    8192), cell groups (other boxes of >= 3 cells per side) or per particle."""
    nc = int(int(box_length(e.n(r))) / 2.85)
    if 2 <= nc <= 4 and e.n(r) <= 8192:
        return "box"
    return "group" if nc >= 3 else "particle"


def autotune(e: Engine, reps: int = 20, verbose: bool = False, mode: str = "forces", step_reps: int = 32) -> dict:
    kinds = {_kind(e, r) for r in range(e.nsys)}

    def measure(label):
        if mode == "step":
            e.bench_steps(step_reps, 0)
            t = e.bench_steps(step_reps, 0)[0] / step_reps
        else:
            e.time_stage(1, 1)
            t = e.time_stage(1, reps)
        if verbose:
            print(f"{label}: {t * 1e3:.1f} us")
        return t

    def pick(label, values, setter):
        best_v, best_t = None, float("inf")
        for val in values:
            setter(val)
            t = measure(f"{label} {val}")
            if t < best_t:
                best_v, best_t = val, t
        setter(best_v)
        return best_v, best_t

    out = {}
    out["group_tpp"], t = pick("group/box tpp", GROUP_TPP, e.set_group_tpp)
    if "box" in kinds:
        out["box_cells"], t = pick("box cells", BOX_CELLS, e.set_box_cells)
    best_s = e.get_launch()
    if "particle" in kinds:
        best_s, t = pick("small-box kernel", SMALL_SHAPES, lambda sh: e.set_launch(*sh))
    out["tpp"], out["block"] = best_s
    out["ms" if mode == "step" else "force_ms"] = t
    out["mode"] = mode
    return out
