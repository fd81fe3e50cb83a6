"""The space-time objective and its gradient in one batched device pass.

For a density field ``xPhys`` on an ``nelx x nely`` grid (bottom node row clamped and
the build plate, self-weight loading, SIMP ``Emin + x^p (E0 - Emin)``):

1. virtual-heat time field: ``-div(chi grad T) + alpha T = 0``, ``T = 1`` on the plate,
   ``chi = max(x^q, 1e-6)`` (``q`` the conduction penalty, ``mu = 1/2``),
   ``alpha = drain_beta / (nelx nely)``; ``t = 1 - T``, element means, normalised over
   the part (sttopt/virtual_heat.py:404-462);
2. stage membership ``m_s = [tPhys <= s / n_stage]`` (bit-exact FP64 compare);
3. all stage solves ``K(x m_s) U_s = F_s`` with ``F_s[y] = -C (x m_s)`` as ONE batched
   device PCG (sttopt/compliance.py:137-161,198-253 with the hard threshold);
4. objective ``sum_s c_s + sum(w tPhys)``;
5. gradient: the stage adjoints (warm-started at ``alpha U``, exact for compliance), the
   element terms and the load-dependence term in one kernel, plus the true adjoint of
   the heat solve on the heat hierarchy.

``precision="mixed"`` runs both V-cycles in FP32 inside the FP64 PCG; ``"fp64"`` runs
everything in FP64.  ``batched=False`` solves the stages one at a time (the plain
form the batched one is compared against).
"""

from __future__ import annotations

from typing import Callable

import torch
from torch import Tensor

from . import _geom, _lib, fem, torch_fem, torch_mg

EMIN, EMAX, PENAL, NU = 1e-9, 1.0, 3.0, 0.3


class SpaceTimeProblem:
    """Grid-level constants of the space-time objective, built once per shape."""

    def __init__(self, nelx: int, nely: int, device, *, nu: float = NU):
        self.nelx, self.nely = nelx, nely
        self.nel = nelx * nely
        self.nnode = (nelx + 1) * (nely + 1)
        self.device = device
        self.KE = torch.tensor(fem.plane_stress_KE(nu), dtype=torch.float64, device=device)
        self.KEh = torch.tensor(fem.diffusion_KE(), dtype=torch.float64, device=device)
        self.edof = torch_mg.element_dof_map_tensor(nelx, nely, device, 2)
        self.edof1 = torch_mg.element_dof_map_tensor(nelx, nely, device, 1)
        nodes = torch.arange(self.nnode, device=device).reshape(nely + 1, nelx + 1)
        plate = torch.zeros(self.nnode, dtype=torch.bool, device=device)
        plate[nodes[-1, :].reshape(-1)] = True
        self.plate = plate
        self.heat_mask = ~plate
        self.mask = (~plate)[:, None].expand(self.nnode, 2).reshape(-1).contiguous()
        self.fixed2 = _geom.fixed_flags(self.mask, self.nnode, 2)
        self.fixed1 = _geom.fixed_flags(self.heat_mask, self.nnode, 1)
        self.lift = plate.to(torch.float64)
        self.ke = _lib.dbl_array(_geom.host_KE(self.KE))
        # 2 KE: the stage adjoint's load 2 K U in one apply (doubling is exact)
        self.ke2 = _lib.dbl_array([2.0 * v for v in _geom.host_KE(self.KE)])
        self.keh = _lib.dbl_array(_geom.host_KE(self.KEh))
        self._streams: dict = {}
        self._worker = None

    def worker(self):
        """A single host thread kept for this problem's lifetime (the heat adjoint's
        driver): creating one per evaluation cost ~0.6 ms of idle GPU a step."""
        if self._worker is None:
            import concurrent.futures

            self._worker = concurrent.futures.ThreadPoolExecutor(max_workers=1)
        return self._worker

    def stream(self, name: str) -> torch.cuda.Stream:
        """A CUDA stream kept for this problem's lifetime.  Side work reuses one stream
        per role across evaluations: torch's caching allocator pools memory per stream,
        so a fresh stream per evaluation would cudaMalloc (and stall) every time."""
        s = self._streams.get(name)
        if s is None:
            s = self._streams[name] = torch.cuda.Stream(device=_device_index(self.device))
        return s


def _pcg(levels, b, x0, rtol, max_iter, info_key, info, x0_inplace=False):
    """The device MG-PCG solve (``x0_inplace``: the warm start's own buffer becomes the
    solution, for the package's warm starts)."""
    M = torch_mg.VCycle(levels)
    sub = {}
    out = levels[0]._native_pcg(b, M, rtol=rtol, max_iter=max_iter, x0=x0, info=sub,
                                x0_inplace=x0_inplace) if x0_inplace else None
    if out is None:
        out = torch_fem.pcg(levels[0], b, M, rtol=rtol, max_iter=max_iter, x0=x0, info=sub)
    x, n = out
    if info is not None:
        info[info_key] = n
    return x


def objective_and_gradient(xPhys: Tensor, w: Tensor, *, n_stage: int = 16, precision: str = "mixed",
                           rtol: float = 1e-8, max_iter: int = 500, drain_beta: float = 25.0,
                           conduction_penal: float = 3.0, Emin: float = EMIN, Emax: float = EMAX,
                           penal: float = PENAL, max_coarse_elements: int = torch_mg.MAX_COARSE_ELEMENTS,
                           gradient: bool = True, batched: bool = True,
                           problem: SpaceTimeProblem | None = None, info: dict | None = None,
                           overlap: bool = True, filter=None, beta: float | None = None,
                           eta: float = 0.5) -> dict:
    """Objective, stage compliances, ``tPhys`` and (optionally) ``d objective / d xPhys``.
    ``overlap`` runs the heat adjoint on a side stream concurrently with the stage work.

    With ``filter`` (``filters.density_filter``'s ``ConeFilter``) the input is the design
    variable x and the physical density is ``xPhys = P(H x / Hs)`` (the Heaviside projection
    with ``beta``, ``eta``; the filter alone when ``beta`` is None), as sttopt/stto_heat.py:177-189
    forms it: one stencil pass gives ``xTilde`` and ``xPhys``, and the gradient is taken
    back to x by one pass of the filter's transpose fused with the projection's derivative,
    ``H (g P'(xTilde) / Hs)``.  The result then also holds ``xPhys``, ``xTilde`` and
    ``gradient_xPhys``."""
    _lib.require_cuda(xPhys, w)
    nely, nelx = xPhys.shape
    P = problem if problem is not None and (problem.nelx, problem.nely) == (nelx, nely) else \
        SpaceTimeProblem(nelx, nely, xPhys.device)
    opts = dict(precision=precision, rtol=rtol, max_iter=max_iter, drain_beta=drain_beta,
                conduction_penal=conduction_penal, Emin=Emin, Emax=Emax, penal=penal,
                max_coarse_elements=max_coarse_elements, gradient=gradient, batched=batched, overlap=overlap)
    if filter is None:
        return _solve_group(P, [xPhys], [w], [n_stage], info=info, **opts)[0]
    from . import filters

    b = 0.0 if beta is None else float(beta)
    xTilde, xp = filters._filter(xPhys, filter, b, float(eta))
    xp = xTilde if xp is None else xp
    out = _solve_group(P, [xp], [w], [n_stage], info=info, **opts)[0]
    out["xPhys"], out["xTilde"] = xp, xTilde
    if gradient:
        out["gradient_xPhys"] = out["gradient"]
        out["gradient"] = filters._adjoint(out["gradient"], filter, xTilde if b > 0 else None, b, float(eta))
    return out


def objective_and_gradient_part(xPhys: Tensor, w: Tensor, *, n_stage: int = 16, stages: list[int],
                                tphys: Tensor | None = None, publish: Callable[[Tensor], None] | None = None,
                                precision: str = "mixed", rtol: float = 1e-8, max_iter: int = 500,
                                drain_beta: float = 25.0, conduction_penal: float = 3.0, Emin: float = EMIN,
                                Emax: float = EMAX, penal: float = PENAL,
                                max_coarse_elements: int = torch_mg.MAX_COARSE_ELEMENTS,
                                problem: SpaceTimeProblem | None = None, info: dict | None = None) -> dict:
    """A rank's share of one objective split over ranks (``sharding.objective_and_gradient_split``):
    the compliances ``c_s`` of ``stages`` (in that order) and their gradient terms, plus,
    when ``tphys`` is None, the heat solve (``publish(tPhys)`` is called as soon as it
    exists) and the heat adjoint's gradient term; with ``tphys`` given, neither."""
    _lib.require_cuda(xPhys, w)
    nely, nelx = xPhys.shape
    P = problem if problem is not None and (problem.nelx, problem.nely) == (nelx, nely) else \
        SpaceTimeProblem(nelx, nely, xPhys.device)
    return _solve_group(P, [xPhys], [w], [n_stage], precision=precision, rtol=rtol, max_iter=max_iter,
                        drain_beta=drain_beta, conduction_penal=conduction_penal, Emin=Emin, Emax=Emax, penal=penal,
                        max_coarse_elements=max_coarse_elements, gradient=True, batched=True, info=info,
                        stage_subset=list(stages), tphys=tphys, publish=publish)[0]


def objective_and_gradient_many(xs: list[Tensor], ws: list[Tensor], n_stages: list[int], *,
                                precision: str = "mixed", rtol: float = 1e-8, max_iter: int = 500,
                                drain_beta: float = 25.0, conduction_penal: float = 3.0,
                                Emin: float = EMIN, Emax: float = EMAX, penal: float = PENAL,
                                max_coarse_elements: int = torch_mg.MAX_COARSE_ELEMENTS,
                                gradient: bool = True, concurrent: bool = True,
                                problems: dict | None = None, info: dict | None = None,
                                memory_budget: int | None = None) -> list[dict]:
    """Many independent space-time problems of uneven grid sizes and stage counts.

    Problems of one grid size form one group: their heat solves are one batched device
    PCG (a row per problem), and all their stage solves and stage adjoints are one
    batched device PCG each (a row per stage, hierarchy rows per stage density).  With
    ``concurrent`` the groups run on their own CUDA streams from host threads, so the
    GPU overlaps them.  Results come back in input order, each as
    ``objective_and_gradient`` returns it.  ``problems`` caches ``SpaceTimeProblem`` per
    shape; ``info`` receives per-group iteration counts under ``(nelx, nely)``.

    ``memory_budget`` (bytes) bounds what the solves hold at once: each group's device
    memory is estimated (``group_bytes``: its hierarchies, solve workspaces and the
    stage rows' vectors), groups over the budget are split into slices of their problems,
    and the slices run in waves whose estimates fit the budget (at most one slice per grid
    size in a wave), one wave after another; without it every group runs at once.
    """
    if not (len(xs) == len(ws) == len(n_stages)):
        raise ValueError("xs, ws and n_stages must have the same length")
    _lib.require_cuda(*xs, *ws)
    opts = dict(precision=precision, rtol=rtol, max_iter=max_iter, drain_beta=drain_beta,
                conduction_penal=conduction_penal, Emin=Emin, Emax=Emax, penal=penal,
                max_coarse_elements=max_coarse_elements, gradient=gradient, batched=True, overlap=True)
    groups: dict = {}
    for k, x in enumerate(xs):
        groups.setdefault(tuple(x.shape), []).append(k)
    cache = problems if problems is not None else {}
    dev = xs[0].device
    for (nely, nelx) in groups:
        if (nelx, nely) not in cache:
            cache[(nelx, nely)] = SpaceTimeProblem(nelx, nely, dev)
    results: list = [None] * len(xs)
    if memory_budget is None:
        waves = [list(groups.items())]
    else:
        waves = budget_waves(groups, n_stages, int(memory_budget), precision, max_coarse_elements)

    def run(shape, idx):
        nely, nelx = shape
        sub = {} if info is not None else None
        out = _solve_group(cache[(nelx, nely)], [xs[k] for k in idx], [ws[k] for k in idx],
                           [n_stages[k] for k in idx], info=sub, **opts)
        if info is not None:
            info.setdefault((nelx, nely), {}).update(sub)
        for k, o in zip(idx, out):
            results[k] = o

    for wave in waves:
        _run_wave(wave, run, cache, dev, concurrent)
    if concurrent and any(len(w) > 1 for w in waves):
        main = torch.cuda.current_stream(_device_index(dev))
        for o in results:  # made on side streams, used on the caller's
            for v in o.values():
                if isinstance(v, torch.Tensor) and v.is_cuda:
                    v.record_stream(main)
    return results


def group_bytes(nelx: int, nely: int, n_problems: int, stage_rows: int, precision: str,
                max_coarse_elements: int = torch_mg.MAX_COARSE_ELEMENTS) -> int:
    """Estimated device bytes of one grid size's batched solves: the stage and heat
    hierarchies (the library's workspace sizes), the solve workspaces (FP64 PCG vectors and
    the cycle's per-level vectors, ~100 bytes a dof) and the group's own vectors (densities,
    loads, U, the adjoint's load, warm start and solution, element terms: ~40 bytes a dof
    and 40 an element), a quarter added for the allocator's rounding."""
    L = _lib.lib()
    prec = _lib.STT_FP32 if precision == "mixed" else _lib.STT_FP64
    nel, nnode = nelx * nely, (nelx + 1) * (nely + 1)
    stage = L.stt_hier_workspace_bytes(2, nelx, nely, stage_rows, max_coarse_elements, prec)
    heat = L.stt_hier_workspace_bytes(1, nelx, nely, n_problems, max_coarse_elements, prec)
    rows = stage_rows * (2 * nnode * 140 + nel * 40) + n_problems * (nnode * 140 + nel * 40)
    return int(1.25 * (stage + heat + rows))


def budget_waves(groups: dict, n_stages, budget: int, precision: str, max_coarse_elements: int) -> list:
    """Slices of the shape groups (``{(nely, nelx): [problem indices]}``) packed into waves
    whose ``group_bytes`` estimates fit ``budget``: a group over the budget is cut into
    slices of consecutive problems that fit (a single problem over the budget is a slice of
    its own); slices go first-fit, largest first, into the first wave with room and no
    slice of the same grid size."""
    slices = []
    for shape, idx in groups.items():
        nely, nelx = shape
        cur: list = []
        for k in idx:
            trial = cur + [k]
            est = group_bytes(nelx, nely, len(trial), sum(n_stages[i] for i in trial), precision, max_coarse_elements)
            if cur and est > budget:
                slices.append((shape, cur))
                cur = [k]
            else:
                cur = trial
        if cur:
            slices.append((shape, cur))

    def est(sl):
        (nely, nelx), idx = sl
        return group_bytes(nelx, nely, len(idx), sum(n_stages[i] for i in idx), precision, max_coarse_elements)

    waves: list = []  # [load, shapes, slices]
    for sl in sorted(slices, key=lambda t: -est(t)):
        e = est(sl)
        for w in waves:
            if w[0] + e <= budget and sl[0] not in w[1]:
                w[0] += e
                w[1].add(sl[0])
                w[2].append(sl)
                break
        else:
            waves.append([e, {sl[0]}, [sl]])
    return [w[2] for w in waves]


def _run_wave(wave: list, run, cache: dict, dev, concurrent: bool) -> None:
    """One wave of ``(shape, problem indices)`` slices: on concurrent CUDA streams from host
    threads (one slice per grid size), or in order on the caller's stream."""
    if not concurrent or len(wave) == 1:
        for shape, idx in wave:
            run(shape, idx)
        return
    import concurrent.futures

    dev_i = _device_index(dev)
    main = torch.cuda.current_stream(dev_i)
    ready = torch.cuda.Event()
    ready.record(main)
    streams = {shape: cache[(shape[1], shape[0])].stream("group") for shape, _ in wave}

    def on_stream(shape, idx):
        torch.cuda.set_device(dev_i)
        s = streams[shape]
        s.wait_event(ready)
        with torch.cuda.stream(s):
            run(shape, idx)
        return s

    with concurrent.futures.ThreadPoolExecutor(max_workers=len(wave)) as ex:
        futs = [ex.submit(on_stream, shape, idx) for shape, idx in wave]
        done = [f.result() for f in futs]
    for s in done:  # the results were made on the side streams
        main.wait_stream(s)


def _device_index(dev) -> int:
    """The CUDA device index of ``dev`` (an index-less "cuda" means the caller's current
    device), for host threads, whose current device is their own."""
    dev = torch.device(dev)
    return dev.index if dev.index is not None else torch.cuda.current_device()


def concurrent_wait(fut) -> None:
    """Waits for a future, dropping its result or error."""
    import concurrent.futures

    concurrent.futures.wait([fut])


class _HeatAdjoint:
    """The heat adjoint solves of a group on a side stream, driven by a host thread.

    d(sum w tPhys)/dT = -(w / scale) / 4 per corner; the adjoint is warm-started at the
    exact multiple of T_free (compliance-like), and -lam_e^T KE_h T_e gives both the
    density term of the solve and the lift term.  ``result()`` joins the thread and
    orders the caller's stream after the side stream."""

    def __init__(self, P, hl, T, T_free, heat_rhs, Ws, rtol, max_iter, info, threaded=True):
        self.dev = _device_index(P.device)
        self.main = torch.cuda.current_stream(self.dev)
        if not threaded:  # in order on the caller's stream
            self.side, self.pool = self.main, None
            self.g_chi = self._run(P, hl, T, T_free, heat_rhs, Ws, rtol, max_iter, info)
            return
        self.side = P.stream("heat_adjoint")
        self.side.wait_stream(self.main)
        self.pool = P.worker()
        self.fut = self.pool.submit(self._run, P, hl, T, T_free, heat_rhs, Ws, rtol, max_iter, info)

    def _run(self, P, hl, T, T_free, heat_rhs, Ws, rtol, max_iter, info):
        torch.cuda.set_device(self.dev)
        with torch.cuda.stream(self.side):
            L, st = _lib.lib(), _lib.stream()
            G, nnode = T.shape
            gT = torch.empty(G, nnode, dtype=torch.float64, device=P.device)
            for g in range(G):
                _lib.check(L.stt_heat_adjoint_load(P.nelx, P.nely, _lib.ptr(Ws[g]), 1.0, _lib.ptr(gT[g]), st))
            gT = torch_fem.project(gT, P.heat_mask).contiguous()
            # T_free . gT and T_free . heat_rhs in one pass over T_free
            Tf, hr = T_free.contiguous(), heat_rhs.contiguous()
            d2 = torch.empty(G, 2, dtype=torch.float64, device=P.device)
            _lib.check(L.stt_vec_dots(G, nnode, _lib.ptr(Tf), _lib.ptr(gT), _lib.ptr(Tf), _lib.ptr(hr), None, None,
                                      nnode, _lib.ptr(d2), st))
            ah = torch_fem.safe_div(d2[:, 0], d2[:, 1])
            lam_h = _pcg(hl, gT, (ah[:, None] * T_free).contiguous(), rtol, max_iter, "heat_adjoint_n_iter", info)
            return torch_fem.element_terms(T, P.edof1, P.KEh, lam=lam_h.reshape(G, nnode))["gdens"]

    def result(self):
        if self.pool is None:
            return self.g_chi
        g_chi = self.fut.result()
        self.main.wait_stream(self.side)
        g_chi.record_stream(self.main)
        return g_chi

    def abandon(self):
        """Wait for the side work and drop it (the caller is unwinding an error)."""
        if self.pool is None:
            return
        concurrent_wait(self.fut)
        self.main.wait_stream(self.side)


def _solve_group(P: SpaceTimeProblem, xs: list[Tensor], ws: list[Tensor], n_stages: list[int], *,
                 precision: str, rtol: float, max_iter: int, drain_beta: float, conduction_penal: float,
                 Emin: float, Emax: float, penal: float, max_coarse_elements: int, gradient: bool,
                 batched: bool, info: dict | None, overlap: bool = True,
                 stage_subset: list[int] | None = None, tphys: Tensor | None = None,
                 publish: Callable[[Tensor], None] | None = None) -> list[dict]:
    """G problems on one grid: batched heat solve, all stage rows in one batched solve.

    For one problem (G = 1) a share of its work, as the ranks of a split objective do it:
    ``stage_subset`` solves only those stages (``c_s`` and the gradient then cover them
    only); ``tphys`` takes the time field as given (no heat solve, no heat adjoint);
    ``publish(tPhys)`` is called as soon as the heat solve has produced it."""
    L = _lib.lib()
    st = _lib.stream()
    nelx, nely, nel, nnode = P.nelx, P.nely, P.nel, P.nnode
    dev = P.device
    G = len(xs)
    if (stage_subset is not None or tphys is not None) and G != 1:
        raise ValueError("stage_subset and tphys apply to a single problem")
    X = torch.stack([x.detach().to(torch.float64).reshape(-1) for x in xs]).contiguous()  # (G, nel)
    W = torch.stack([w.detach().to(torch.float64).reshape(-1) for w in ws]).contiguous()
    if tphys is not None:
        return _stage_work(P, X, W, tphys.detach().to(torch.float64).reshape(1, nel).contiguous(), None, n_stages,
                           stage_subset, precision=precision, rtol=rtol, max_iter=max_iter, Emin=Emin, Emax=Emax,
                           penal=penal, max_coarse_elements=max_coarse_elements, gradient=gradient, batched=batched,
                           info=info, conduction_penal=conduction_penal, T=None)

    # 1. heat time fields (a row per problem)
    chi = torch.clamp(X ** conduction_penal, min=1e-6).contiguous()
    alpha = drain_beta / (nelx * nely)
    reac = torch.full_like(chi, alpha)
    hl = torch_mg.build_hierarchy(chi, P.edof1, P.KEh, P.heat_mask, nelx, nely, reaction=reac,
                                  max_coarse_elements=max_coarse_elements, precision=precision, check=False)
    rdiag = hl[0].reaction_diag.reshape(G, nnode).contiguous()
    Klift = torch.empty(G, nnode, dtype=torch.float64, device=dev)
    _lib.check(L.stt_q4_apply(_lib.STT_FP64, 1, nelx, nely, G, _lib.ptr(P.lift), 0, _lib.ptr(Klift),
                              nnode, _lib.ptr(chi), nel, _lib.ptr(rdiag), nnode, _lib.ptr(P.fixed1),
                              _lib.STT_PROJECT_OUT, P.keh, st))
    heat_rhs = (-Klift).contiguous()  # F - K_lift, projected (F = 0)
    T_free = _pcg(hl, heat_rhs, None, rtol, max_iter, "heat_n_iter", info).reshape(G, nnode)
    T = (T_free + P.lift).contiguous()
    t_e = torch.empty(G, nel, dtype=torch.float64, device=dev)
    for g in range(G):
        _lib.check(L.stt_heat_element_means(nelx, nely, _lib.ptr(T[g]), _lib.ptr(t_e[g]), st))
    part = X >= X.max(dim=1, keepdim=True).values / 2
    scale = torch.where(part, t_e, torch.full_like(t_e, -torch.inf)).max(dim=1, keepdim=True).values
    tPhys = (t_e / scale).contiguous()
    if publish is not None:
        publish(tPhys[0])

    # 5b (overlapped). The heat adjoints need only T, tPhys's scale and w, not the stage
    # solves: they run from a host thread on a side stream while this thread launches the
    # stage work, so the heat solve's small, latency-bound kernels fill gaps in the
    # bandwidth-bound stage kernels instead of adding to the step.
    heat_adj = None
    if gradient:
        heat_adj = _HeatAdjoint(P, hl, T, T_free, heat_rhs, (W / scale).contiguous(), rtol, max_iter, info,
                                threaded=overlap)

    try:
        return _stage_work(P, X, W, tPhys, heat_adj, n_stages, stage_subset, precision=precision, rtol=rtol,
                           max_iter=max_iter, Emin=Emin, Emax=Emax, penal=penal,
                           max_coarse_elements=max_coarse_elements, gradient=gradient, batched=batched, info=info,
                           conduction_penal=conduction_penal, T=T)
    except BaseException:
        if heat_adj is not None:
            heat_adj.abandon()
        raise


def _heat_share(heat_adj, X: Tensor, conduction_penal: float, grads: Tensor) -> Tensor:
    """``grads`` plus the heat adjoints' share of the gradient (none without a heat adjoint:
    a split objective's ranks that were given the time field)."""
    if heat_adj is None:
        return grads
    g_chi = heat_adj.result()
    q = conduction_penal
    dpen = torch.where(X ** q >= 1e-6, q * X ** (q - 1), torch.zeros_like(X))
    return grads + g_chi * dpen


def _stage_work(P: SpaceTimeProblem, X: Tensor, W: Tensor, tPhys: Tensor, heat_adj, n_stages: list[int],
                stage_subset: list[int] | None, *, precision: str, rtol: float, max_iter: int, Emin: float,
                Emax: float, penal: float, max_coarse_elements: int, gradient: bool, batched: bool,
                info: dict | None, conduction_penal: float, T: Tensor | None) -> list[dict]:
    """Stage membership, the batched stage solves, their adjoints and the gradient (plus
    the heat adjoints' share when ``heat_adj`` is given); ``stage_subset`` (one problem)
    restricts the stages solved."""
    # 2.-3. stage rows of every problem, then the batched stage solves
    L = _lib.lib()
    st = _lib.stream()
    nelx, nely, nel, nnode = P.nelx, P.nely, P.nel, P.nnode
    dev = P.device
    G = X.shape[0]
    counts = list(n_stages) if stage_subset is None else [len(stage_subset)]
    offs = [0]
    for n in counts:
        offs.append(offs[-1] + n)
    S = offs[-1]
    members = []
    rho = torch.empty(S, nel, dtype=torch.float64, device=dev)
    F = torch.empty(S, 2 * nnode, dtype=torch.float64, device=dev)
    for g, n in enumerate(n_stages):
        m = torch.empty(n, nel, dtype=torch.uint8, device=dev)
        _lib.check(L.stt_stage_membership(nel, n, _lib.ptr(tPhys[g]), _lib.ptr(m), st))
        if stage_subset is not None:
            m = m[list(stage_subset)].contiguous()
        if m.shape[0]:
            _lib.check(L.stt_stage_rows(nelx, nely, m.shape[0], _lib.ptr(X[g]), _lib.ptr(m), Emin, Emax, penal,
                                        _lib.ptr(P.fixed2), _lib.ptr(rho[offs[g]]), _lib.ptr(F[offs[g]]), st))
        members.append(m)
    if S == 0:  # a share with no stage rows (more ranks than stages)
        J_t = (W * tPhys).sum(-1)
        outs = [dict(objective=J_t[g], c_s=rho.new_zeros(0), J_t=J_t[g], tPhys=tPhys[g].reshape(nely, nelx), U=F,
                     T=None if T is None else T[g], member=members[g]) for g in range(G)]
        if gradient:
            grads = _heat_share(heat_adj, X, conduction_penal, torch.zeros(G, nel, dtype=torch.float64, device=dev))
            for g in range(G):
                outs[g]["gradient"] = grads[g].reshape(nely, nelx)
                outs[g]["lam"] = F
        return outs
    if batched:
        sl = torch_mg.build_hierarchy(rho, P.edof, P.KE, P.mask, nelx, nely,
                                      max_coarse_elements=max_coarse_elements, precision=precision, check=False)
        U = _pcg(sl, F, None, rtol, max_iter, "stage_n_iter", info)
        stage_levels = [sl]
    else:
        Us, stage_levels = [], []
        for s in range(S):
            sl = torch_mg.build_hierarchy(rho[s], P.edof, P.KE, P.mask, nelx, nely,
                                          max_coarse_elements=max_coarse_elements, precision=precision, check=False)
            Us.append(_pcg(sl, F[s], None, rtol, max_iter, f"stage{s}_n_iter", info))
            stage_levels.append(sl)
        U = torch.stack(Us)
    ce = torch_fem.element_terms(U, P.edof, P.KE)["ce"]
    c_s = torch_fem._dots(rho, ce)
    J_t = (W * tPhys).sum(-1)  # (G rows of nel: one row is too small for the cluster dot kernel)
    outs = []
    for g in range(G):
        a, b = offs[g], offs[g + 1]
        outs.append(dict(objective=c_s[a:b].sum() + J_t[g], c_s=c_s[a:b], J_t=J_t[g],
                         tPhys=tPhys[g].reshape(nely, nelx), U=U[a:b], T=None if T is None else T[g],
                         member=members[g]))
    if not gradient:
        return outs

    # 5a. stage adjoints: dL/dU = 2 K U (one apply with 2 KE), with the warm-start factor's
    # dots U . gK and U . F in the same pass over U; the warm start alpha U (exact for
    # compliance) is written where the adjoint solve starts
    gK = torch.empty_like(U)
    d2 = torch.empty(S, 2, dtype=torch.float64, device=dev)
    ws = _lib.workspace(L.stt_q4_apply_dots_workspace_bytes(nelx, nely, S), dev)
    _lib.check(L.stt_q4_apply_dots(2, nelx, nely, S, _lib.ptr(U), 2 * nnode, _lib.ptr(gK), 2 * nnode,
                                   _lib.ptr(rho), nel, _lib.ptr(P.fixed2), P.ke2, _lib.ptr(F), 2 * nnode,
                                   _lib.ptr(d2), _lib.ptr(ws), ws.numel(), st))
    x0 = torch.empty_like(U)
    _lib.check(L.stt_adjoint_warm_start(S, 2 * nnode, _lib.ptr(d2), _lib.ptr(U), 2 * nnode, _lib.ptr(x0),
                                        2 * nnode, st))
    if batched:
        lam = _pcg(stage_levels[0], gK, x0, rtol, max_iter, "adjoint_n_iter", info, x0_inplace=True)
    else:
        lam = torch.stack([_pcg(stage_levels[s], gK[s], x0[s], rtol, max_iter, f"adjoint{s}_n_iter", info)
                           for s in range(S)])
    lam = lam.contiguous()
    gd = torch_fem.element_terms(U, P.edof, P.KE, lam=lam)["gdens"]
    grads = torch.zeros(G, nel, dtype=torch.float64, device=dev)
    for g, n in enumerate(counts):
        a = offs[g]
        _lib.check(L.stt_stage_gradient(nelx, nely, n, _lib.ptr(X[g]), _lib.ptr(members[g]), _lib.ptr(ce[a]),
                                        _lib.ptr(gd[a]), _lib.ptr(lam[a]), Emin, Emax, penal,
                                        _lib.ptr(grads[g]), st))

    # 5b. the heat adjoints' share of the gradient
    grads = _heat_share(heat_adj, X, conduction_penal, grads)
    for g in range(G):
        outs[g]["gradient"] = grads[g].reshape(nely, nelx)
        outs[g]["lam"] = lam[offs[g]:offs[g + 1]]
    return outs


class _HeatConfig:
    """The fields of ``HeatRunConfig`` that ``heat_time_field`` reads (sttopt/run_config.py:495)."""

    def __init__(self, drain_beta: float, rtol: float):
        self.chi_contrast = 1000.0  # mu = 1/2 makes chi's contrast factor 1
        self.drain_beta = drain_beta
        self.time_map = "one_minus"
        self.heat_cg_rtol = rtol


class DropInChain:
    """The space-time objective composed only of the reference-signature functions, as a
    caller of the reference would write it (sttopt/stto_heat.py:192-327 with the hard stage
    threshold): ``virtual_heat.heat_time_field`` -> ``compliance.batched_whole_and_gravity_compliance``
    (``mask_fn=hard_time_mask``, the whole-structure row unloaded) -> ``sum_s c_s + sum(w tPhys)``
    -> ``sensitivity.jacobian_rows``.  The grid-level set-up (meshes, element matrices, the
    build-plate clamp, the gravity stencil) is built once.  ``precision="mixed"`` routes
    the stage solve through the ``_solve_fe_batched`` patch point with the FP32 V-cycle
    (and the heat solve likewise); ``"fp64"`` is the reference's arithmetic."""

    def __init__(self, nelx: int, nely: int, device, *, n_stage: int = 16, drain_beta: float = 25.0,
                 rtol: float = 1e-8, conduction_penal: float = 3.0):
        from . import gravity, load_cases, virtual_heat

        self.nelx, self.nely, self.n_stage = nelx, nely, n_stage
        self.mesh = virtual_heat.ScalarMesh.build(nelx, nely, "bottom_edge", device, torch.float64)
        self.cfg = _HeatConfig(drain_beta, rtol)
        self.rtol = rtol
        self.conduction_penal = conduction_penal
        self.KE = torch.tensor(fem.plane_stress_KE(NU), dtype=torch.float64, device=device)
        self.edof = torch_mg.element_dof_map_tensor(nelx, nely, device, 2)
        F, free = load_cases.build_plate_clamp(nelx, nely)
        self.F = torch.as_tensor(F, device=device)
        self.free = torch.as_tensor(free, device=device)
        self.ndof = F.size
        self.C = gravity.gravity_load_matrix(nelx, nely)
        self.mu = torch.full((nely, nelx), 0.5, dtype=torch.float64, device=device)
        self.times = [s / n_stage for s in range(1, n_stage + 1)]

    def __call__(self, xPhys: Tensor, w: Tensor, precision: str = "fp64") -> dict:
        from . import compliance, sensitivity, torch_solve, virtual_heat

        x = xPhys.detach().to(torch.float64).requires_grad_(True)
        prec = None if precision == "fp64" else precision
        sol = virtual_heat.heat_time_field(self.cfg, self.mesh, x, self.mu, conduction_penal=self.conduction_penal,
                                           precision=prec)
        patched = None
        if prec is not None:
            rtol = self.rtol

            def solve_fe_batched(KE, density, edofMat, mask, nelx, nely, F, *, x0=None):
                return torch_solve.femsolve(density, F, edofMat, KE, mask, nelx, nely, x0=x0, rtol=rtol,
                                            precision=prec)

            patched = compliance._solve_fe_batched
            compliance._solve_fe_batched = solve_fe_batched
        try:
            c, stages, U = compliance.batched_whole_and_gravity_compliance(
                x, sol.tPhys, self.KE, self.edof, EMIN, EMAX, PENAL, self.free, self.F, self.ndof, self.C, 1.0,
                self.times, mask_fn=compliance.hard_time_mask)
        finally:
            if patched is not None:
                compliance._solve_fe_batched = patched
        c_s = torch.stack(stages)
        L = c_s.sum() + torch.sum(w * sol.tPhys)
        (g,) = sensitivity.jacobian_rows(L[None], [x])
        return dict(objective=L.detach(), c_s=c_s.detach(), tPhys=sol.tPhys.detach(), U=U.detach()[1:],
                    gradient=g.reshape(self.nely, self.nelx))


class SpaceTimeObjective(torch.autograd.Function):
    """``objective(xPhys)`` as an autograd node: the forward pass runs the batched solves
    and the hand-written adjoints at once (``objective_and_gradient``); the backward
    pass scales the stored gradient, so ``torch.autograd.grad`` and
    ``sensitivity.jacobian_rows`` see the space-time objective like any torch function
    (the reference reaches it through autograd over compliance.py and
    virtual_heat.py)."""

    @staticmethod
    def forward(ctx, xPhys, w, kw):
        out = objective_and_gradient(xPhys, w, gradient=ctx.needs_input_grad[0], **kw)
        ctx.save_for_backward(out.get("gradient", torch.zeros_like(xPhys)))
        return out["objective"].clone()

    @staticmethod
    def backward(ctx, g):
        (grad,) = ctx.saved_tensors
        return g * grad.to(g.dtype), None, None


def objective(xPhys: Tensor, w: Tensor, **kw) -> Tensor:
    """Differentiable space-time objective ``sum_s c_s + sum(w tPhys)`` (a 0-d tensor);
    keyword arguments as ``objective_and_gradient``."""
    return SpaceTimeObjective.apply(xPhys, w, kw)
