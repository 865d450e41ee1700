"""Ensembles of oil-water realisations on the GPU.

`run_ensemble`, `EnsembleResult` and `gaussian_samples` keep the interface
of pymrst/modules/ensemble/ensemble_impl.py:17-67.  The reference runs the
members one after another; here `run_ensemble` splits the members over the
ranks of an initialised process group (contiguous blocks balanced by a cost
such as the cell count, no communication until one gather of the results).

`GpuOilWaterEnsemble` runs many oil-water realisations as ONE device model:
their grids are stored side by side as a model whose members share no
interface, so every assembly, SpMV, AMG and smoother launch covers all
members at once.  Newton convergence, the update and timestep cuts stay per
member (pmb_ow_step_members): a converged member is frozen while the others
iterate, and a member that must cut its step repeats it alone, as
`simulate_schedule_ad` (pymrst/modules/ad_core/simulators/
simulate_schedule_ad.py:45-75) would for that member.  The members share the
fluid, gravity and solver options; each has its own grid, rock and wells.
"""

from __future__ import annotations

from dataclasses import dataclass
from types import SimpleNamespace
from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np

from . import _native as N
from .ow_model import GpuOilWaterModel, OWState, _torch, default_cpr_options, face_transmissibility_device
from .params import fluid_params, pore_volume


# -- the reference's ensemble interface (ensemble_impl.py:17-67) ----------------------

@dataclass
class EnsembleResult:
    """Members' parameters, shape (n_par, N), and quantities of interest,
    shape (n_obs, N): one column per member.  The statistics run across the
    members (axis 1); the spread is the sample standard deviation."""

    parameters: np.ndarray
    qoi: np.ndarray

    @property
    def mean(self) -> np.ndarray:
        return np.mean(self.qoi, axis=1)

    @property
    def std(self) -> np.ndarray:
        n = self.qoi.shape[1]
        dev = self.qoi - self.mean[:, None]
        return np.sqrt(np.sum(dev * dev, axis=1) / (n - 1))

    def percentile(self, q) -> np.ndarray:
        return np.percentile(self.qoi, q, axis=1)


def gaussian_samples(mean: np.ndarray, cov: np.ndarray, n: int,
                     rng: Optional[np.random.Generator] = None) -> np.ndarray:
    """n draws of N(mean, cov) as the columns of an (n_par, n) array; `cov`
    may be given as its diagonal.  Each column is mean + L z with L the lower
    Cholesky factor of cov and z a column of standard normals drawn as one
    (n_par, n) block, so a generator in a given state yields the same
    ensemble as the reference's sampler does."""
    gen = rng if rng is not None else np.random.default_rng()
    mu = np.ravel(np.asarray(mean, dtype=float))
    c = np.asarray(cov, dtype=float)
    L = np.linalg.cholesky(np.diag(c) if c.ndim == 1 else c)
    z = gen.standard_normal((mu.size, n))
    return L @ z + mu[:, None]


def shard_members(costs: Sequence[float], world: int) -> List[Tuple[int, int]]:
    """Contiguous blocks [start, stop) of members, one per rank, with the
    cumulative cost split as evenly as block boundaries allow."""
    costs = np.asarray(costs, float)
    n = costs.size
    if world < 1:
        raise ValueError("world size must be positive")
    cum = np.concatenate([[0.0], np.cumsum(costs)])
    total = cum[-1]
    bounds = [0]
    for r in range(1, world):
        target = total * r / world
        b = int(np.searchsorted(cum, target, side="left"))
        if b > 0 and abs(cum[b - 1] - target) <= abs(cum[b] - target):
            b -= 1
        bounds.append(min(max(b, bounds[-1]), n))
    bounds.append(n)
    return [(bounds[r], bounds[r + 1]) for r in range(world)]


def run_ensemble(parameters: np.ndarray, simulate: Callable[[np.ndarray], np.ndarray],
                 costs: Optional[Sequence[float]] = None) -> EnsembleResult:
    """Run `simulate` once per member (run_ensemble, ensemble_impl.py:49-67).

    Under an initialised torch.distributed process group each rank runs its
    contiguous block of members (balanced by `costs`, default equal) and the
    results are gathered on every rank."""
    m = np.atleast_2d(np.asarray(parameters, float))
    nmem = m.shape[1]
    rank, world = 0, 1
    try:
        import torch.distributed as dist
        if dist.is_available() and dist.is_initialized():
            rank, world = dist.get_rank(), dist.get_world_size()
    except ImportError:
        dist = None
    blocks = shard_members(np.ones(nmem) if costs is None else costs, world)
    lo, hi = blocks[rank]
    local = [(k, np.asarray(simulate(m[:, k]), float).ravel()) for k in range(lo, hi)]
    if world > 1:
        gathered = [None] * world
        dist.all_gather_object(gathered, local)
        local = [item for part in gathered for item in part]
    cols = [c for _, c in sorted(local, key=lambda kc: kc[0])]
    lengths = sorted({c.size for c in cols})
    if len(lengths) > 1:
        raise ValueError(f"every member must return a quantity of interest of one length; got {lengths}")
    return EnsembleResult(parameters=m, qoi=np.column_stack(cols))


# -- batched realisations on the device ------------------------------------------

class GpuOilWaterEnsemble(GpuOilWaterModel):
    """Many oil-water realisations (grid, rock, wells each) as one device
    model with per-member Newton convergence and timestep cuts."""

    def __init__(self, members: Sequence[Tuple], fluid, gravity: float = 0.0, ds_max: float = 0.2,
                 dp_max_rel: float = 0.2, tol_cnv: float = 1e-3, tol_mb: float = 1e-7, tol_well: float = 1e-6,
                 max_iterations: int = 25, cpr_options: Optional[dict] = None):
        torch = _torch()
        if not members:
            raise ValueError("an ensemble needs at least one member")
        self.fluid = fluid
        self.raw_fluid = fluid
        self.gravity = float(gravity)
        self.ds_max, self.dp_max_rel = float(ds_max), float(dp_max_rel)
        self.tol_cnv, self.tol_mb, self.tol_well = float(tol_cnv), float(tol_mb), float(tol_well)
        self.max_iterations = int(max_iterations)
        self.linear_solver = None
        prm = fluid_params(fluid)
        self.fluid_params = prm
        Ns, Ts, gdzs, pvs, lines, wells = [], [], [], [], [], []
        cell_ptr, well_ptr = [0], [0]
        self.member_wells: List[list] = []
        for g, rock, mw in members:
            off = cell_ptr[-1]
            nbr = np.asarray(g.faces.neighbors, dtype=np.int64)
            internal = np.all(nbr >= 0, axis=1)
            Nm = nbr[internal]
            tf, _ = face_transmissibility_device(g, rock)
            Ts.append(np.asarray(tf, float)[internal])
            Ns.append(Nm + off)
            if self.gravity:
                z = np.asarray(g.cells.centroids)[:, -1]
                gdzs.append(self.gravity * (z[Nm[:, 1]] - z[Nm[:, 0]]))
            else:
                gdzs.append(np.zeros(Nm.shape[0]))
            pvs.append(pore_volume(g, rock))
            nrm = np.abs(np.asarray(g.faces.normals)[internal])
            lines.append((nrm[:, 2] > nrm[:, 0]) & (nrm[:, 2] > nrm[:, 1]) if nrm.shape[1] == 3
                         else np.zeros(Nm.shape[0], bool))
            mw = list(mw)
            for w in mw:
                if np.asarray(w.compi).size < 2:
                    raise ValueError("wells need 2-phase compi")
                wells.append(SimpleNamespace(cells=np.asarray(w.cells, np.int64).ravel() + off, WI=w.WI, dZ=w.dZ,
                                             compi=w.compi, type=w.type, val=w.val,
                                             refDepth=getattr(w, "refDepth", 0.0)))
            self.member_wells.append(mw)
            cell_ptr.append(off + int(g.cells.num))
            well_ptr.append(well_ptr[-1] + len(mw))
        self.nmembers = len(members)
        self.cell_ptr = np.asarray(cell_ptr, dtype=np.int32)
        self.well_ptr = np.asarray(well_ptr, dtype=np.int32)
        self.N = np.concatenate(Ns)
        self.T = np.concatenate(Ts)
        self.gdz = np.concatenate(gdzs)
        self.pv = np.concatenate(pvs)
        self._line_face = np.concatenate(lines)
        self.wells = wells
        self.nc = int(cell_ptr[-1])
        self.nw = len(wells)
        self.g = SimpleNamespace(cells=SimpleNamespace(num=self.nc))
        self.rock = None
        self._build_handle(prm)
        self.cpr_options = default_cpr_options(**(cpr_options or {}))
        self._cpr = None
        self._stream = torch.cuda.current_stream()

    # -- member states -------------------------------------------------------
    def member_initial_state(self, k: int, p0: float, sw0: float) -> OWState:
        nc = int(self.cell_ptr[k + 1] - self.cell_ptr[k])
        ws = self.member_wells[k]
        return OWState(
            pressure=np.full(nc, float(p0)), sW=np.full(nc, float(sw0)),
            qWs=np.array([float(w.val) * float(np.ravel(w.compi)[0]) if str(w.type).lower() == "rate" else 0.0
                          for w in ws]),
            qOs=np.array([float(w.val) * float(np.ravel(w.compi)[1]) if str(w.type).lower() == "rate" else 0.0
                          for w in ws]),
            bhp=np.array([float(w.val) if str(w.type).lower() == "bhp" else float(p0) for w in ws]))

    def join(self, states: Sequence[OWState]) -> OWState:
        """The batch state from one state per member."""
        return OWState(*(np.concatenate([np.asarray(getattr(s, f), float) for s in states])
                         for f in ("pressure", "sW", "qWs", "qOs", "bhp")))

    def split(self, st: OWState) -> List[OWState]:
        out = []
        for k in range(self.nmembers):
            c0, c1 = self.cell_ptr[k], self.cell_ptr[k + 1]
            w0, w1 = self.well_ptr[k], self.well_ptr[k + 1]
            out.append(OWState(pressure=st.pressure[c0:c1].copy(), sW=st.sW[c0:c1].copy(),
                               qWs=st.qWs[w0:w1].copy(), qOs=st.qOs[w0:w1].copy(), bhp=st.bhp[w0:w1].copy()))
        return out

    # -- stepping --------------------------------------------------------------
    def step_members(self, x, dt: float, active: np.ndarray):
        """One step of the members flagged in `active` on the device state
        `x` (in place).  Returns (state per member: 1 converged, 0 failed and
        restored, -1 untouched; Newton iterations per member; stats4)."""
        state = np.ascontiguousarray(np.where(np.asarray(active, bool), 1, 0), dtype=np.int32)
        its = np.zeros(self.nmembers, dtype=np.int32)
        stats = (N.C.c_double * 4)()
        N.check(N.lib().pmb_ow_step_members(self._handle, self.solver_handle(), N.ptr(x), float(dt),
                                            self.max_iterations, self.nmembers,
                                            N.as_p(self.cell_ptr, N.C.c_int32), N.as_p(self.well_ptr, N.C.c_int32),
                                            N.as_p(state, N.C.c_int32), N.as_p(its, N.C.c_int32), stats))
        return state, its, list(stats)

    def simulate(self, states0: Sequence[OWState], timesteps: Sequence[float], max_cuts: int = 6):
        """Every member through the report steps, with the cut and regrowth
        rule of simulate_schedule_ad applied to each member on its own.
        Returns (states[member][step], iterations[member, step])."""
        nmem = self.nmembers
        x = self.to_device(self.join(states0))
        out: List[List[OWState]] = [[] for _ in range(nmem)]
        its_all = np.zeros((nmem, len(timesteps)), dtype=np.int64)
        self.last_krylov = 0.0
        for i, dt_report in enumerate(timesteps):
            dt_report = float(dt_report)
            t_local = np.zeros(nmem)
            dt = np.full(nmem, dt_report)
            cuts = np.zeros(nmem, dtype=np.int64)
            done = np.zeros(nmem, bool)
            while not done.all():
                dt = np.where(done, dt, np.minimum(dt, dt_report - t_local))
                # members that take the same step size go together
                for h in np.unique(dt[~done]):
                    group = (~done) & (dt == h)
                    state, its, stats = self.step_members(x, float(h), group)
                    self.last_krylov += stats[0]
                    its_all[group, i] += its[group]
                    ok = group & (state == 1)
                    bad = group & (state == 0)
                    t_local[ok] += h
                    dt[ok] = np.where(cuts[ok] > 0, np.minimum(2.0 * h, dt_report - t_local[ok]), dt[ok])
                    cuts[bad] += 1
                    if (cuts > max_cuts).any():
                        k = int(np.flatnonzero(cuts > max_cuts)[0])
                        raise AssertionError(f"member {k}, step {i}: Newton failed after {max_cuts} timestep cuts")
                    dt[bad] = dt[bad] / 2.0
                    done |= ok & (t_local >= dt_report - 1e-12 * dt_report)
            for k, s in enumerate(self.split(self.from_device(x))):
                out[k].append(s)
        return out, its_all


def simulate_members_concurrently(members: Sequence, fluid, states0: Sequence[OWState], timesteps: Sequence[float],
                                  gravity: float = 0.0, workers: int = 16, max_cuts: int = 6,
                                  model_options: Optional[dict] = None, replay_graph: bool = False):
    """Every member on its own device model, `workers` host threads each
    stepping members on its own CUDA stream; each member follows exactly the
    single-run path (simulate_schedule_ad), so its results are those of a
    single run.  `members` are (grid, rock, wells).  Returns
    (states[member][step], iterations[member, step]).

    replay_graph=False launches each member's preconditioner kernel by
    kernel, building and releasing the models inside the threads.  With
    replay_graph=True every model is built before any thread steps and kept
    until all have finished, so that no thread allocates or frees device
    memory (which synchronises the device) while another captures its
    preconditioner graph; the preconditioner is then replayed as a graph.  A
    capture that is disturbed all the same falls back to direct launches for
    that application."""
    import threading
    from concurrent.futures import ThreadPoolExecutor
    from .schedule import simulate_schedule_ad
    torch = _torch()
    opts = dict(model_options or {})
    opts["cpr_options"] = dict(opts.get("cpr_options") or {}, replay_graph=int(bool(replay_graph)))
    workers = max(1, min(int(workers), len(members)))
    if replay_graph:
        streams = [torch.cuda.Stream() for _ in range(workers)]
        models = []
        for k, (g, rock, wells) in enumerate(members):
            with torch.cuda.stream(streams[k % workers]):
                models.append(GpuOilWaterModel(g, rock, fluid, wells, gravity=gravity, **opts))
        torch.cuda.synchronize()

        def run_share(w):
            out = {}
            with torch.cuda.stream(streams[w]):
                for k in range(w, len(members), workers):
                    out[k] = simulate_schedule_ad(states0[k], models[k], timesteps, max_cuts=max_cuts,
                                                  verbose=False)
                streams[w].synchronize()
            return out

        with ThreadPoolExecutor(max_workers=workers) as pool:
            parts = list(pool.map(run_share, range(workers)))
        torch.cuda.synchronize()
        del models
        merged = {k: v for part in parts for k, v in part.items()}
        results = [merged[k] for k in range(len(members))]
        return [r[0] for r in results], np.array([r[1] for r in results])
    local = threading.local()

    def run(k):
        if not hasattr(local, "stream"):
            local.stream = torch.cuda.Stream()
        g, rock, wells = members[k]
        with torch.cuda.stream(local.stream):
            m = GpuOilWaterModel(g, rock, fluid, wells, gravity=gravity, **opts)
            states, its = simulate_schedule_ad(states0[k], m, timesteps, max_cuts=max_cuts, verbose=False)
            local.stream.synchronize()
            del m
        return states, its

    with ThreadPoolExecutor(max_workers=workers) as pool:
        results = list(pool.map(run, range(len(members))))
    return [r[0] for r in results], np.array([r[1] for r in results])


# -- autotuning of the concurrent runner ---------------------------------------------------

def _tune_cache_path():
    import os
    from pathlib import Path
    p = os.environ.get("PMB_TUNE_CACHE")
    if p:
        return Path(p)
    base = os.environ.get("XDG_CACHE_HOME") or os.path.join(os.path.expanduser("~"), ".cache")
    return Path(base) / "pymrst_b200" / "autotune.json"


def tune_key(members, sm_count: int, replay_graph: bool) -> str:
    """Cache key: SM count, graph replay, and the ensemble's shape as powers
    of two (member count, mean cells per member)."""
    n = len(members)
    cells = float(np.mean([m[0].cells.num for m in members])) if n else 0.0
    b = lambda v: int(np.ceil(np.log2(max(v, 1.0))))
    return f"ensemble_workers/sm{sm_count}/graph{int(bool(replay_graph))}/m2^{b(n)}/c2^{b(cells)}"


def tune_workers(members: Sequence, fluid, states0: Sequence[OWState], timesteps: Sequence[float],
                 gravity: float = 0.0, candidates=(4, 8, 16, 32), sample: int = 64, replay_graph: bool = True,
                 model_options: Optional[dict] = None, refresh: bool = False) -> dict:
    """The number of host threads (each with its own stream) for
    simulate_members_concurrently: every candidate runs the first report
    step of a sample of the members (wall clock between device
    synchronisations), and the fastest is cached in a JSON file keyed by
    `tune_key` (PMB_TUNE_CACHE, else the user's cache folder).  Returns
    {"workers", "key", "trials" (seconds per candidate, empty when cached)}."""
    import json
    import time
    torch = _torch()
    sm = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    key = tune_key(members, sm, replay_graph)
    path = _tune_cache_path()
    cache = {}
    if path.exists():
        try:
            cache = json.loads(path.read_text())
        except (OSError, ValueError):
            cache = {}
    if key in cache and not refresh:
        return {"workers": int(cache[key]["workers"]), "key": key, "trials": {}}
    k = max(1, min(int(sample), len(members)))
    trials = {}
    for w in candidates:
        w = int(w)
        if w > k:
            continue
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        simulate_members_concurrently(members[:k], fluid, states0[:k], list(timesteps)[:1], gravity=gravity,
                                      workers=w, model_options=model_options, replay_graph=replay_graph)
        torch.cuda.synchronize()
        trials[w] = time.perf_counter() - t0
    best = min(trials, key=trials.get) if trials else 1
    cache[key] = {"workers": best, "trials": {str(a): b for a, b in trials.items()}}
    try:
        path.parent.mkdir(parents=True, exist_ok=True)
        path.write_text(json.dumps(cache, indent=1, sort_keys=True))
    except OSError:
        pass
    return {"workers": best, "key": key, "trials": trials}
