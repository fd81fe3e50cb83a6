"""Generate the golden fixtures in this folder by running the reference ``sttopt``.

The reference is pure Python (torch + NumPy/SciPy); its own LFS fixtures are absent,
so its FP64 CPU torch path is run here, seeded, and its outputs saved as ``.npz``.
Run from the repository root with the path of a reference checkout, either in the
``REFERENCE_ROOT`` environment variable or as ``--reference PATH``::

    python tests/golden/make_golden.py --reference PATH [--only NAME,NAME] [--with-512] [--full-size]

``--full-size`` adds the benchmark-size fixtures (config 2 at 1024x512, the space-time
objective at 1024x512 and 2048x1024 x 16 stages); the 2048x1024 run takes about ten
minutes and ~20 GB of host memory.  Large fields are stored as seeded random
projections and a strided subsample (``field_summary``), small ones whole.

The fixtures are inputs and outputs only; nothing here is imported at test time.
"""

from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def _reference_root() -> Path:
    if "--reference" in sys.argv:
        return Path(sys.argv[sys.argv.index("--reference") + 1])
    if "REFERENCE_ROOT" in os.environ:
        return Path(os.environ["REFERENCE_ROOT"])
    raise SystemExit("make_golden.py: give the reference checkout as --reference PATH or REFERENCE_ROOT")


REFERENCE_ROOT = _reference_root()
sys.path.insert(0, str(REFERENCE_ROOT))
sys.path.insert(0, str(HERE.parents[1]))

import torch  # noqa: E402

import sttopt.compliance as compliance  # noqa: E402
import sttopt.filters as filters  # noqa: E402
import sttopt.fem as fem  # noqa: E402
import sttopt.gravity as gravity  # noqa: E402
import sttopt.load_cases as load_cases  # noqa: E402
import sttopt.sensitivity as sensitivity  # noqa: E402
import sttopt.torch_fem as torch_fem  # noqa: E402
import sttopt.torch_mg as torch_mg  # noqa: E402
import sttopt.torch_solve as torch_solve  # noqa: E402
import sttopt.torch_util as torch_util  # noqa: E402
import sttopt.virtual_heat as vh  # noqa: E402
from sttopt.run_config import HeatRunConfig  # noqa: E402

from oracle.sttopt_oracle import smoothed_density  # noqa: E402  (seeded input recipe)
sys.path.insert(0, str(HERE))
from summary import field_summary  # noqa: E402

F64 = torch.float64
EMIN, EMAX, PENAL, NU = 1e-9, 1.0, 3.0, 0.3


def t(a, dtype=F64):
    return torch.as_tensor(np.asarray(a), dtype=dtype)


def save(name, **arrays):
    out = {k: (v.detach().cpu().numpy() if torch.is_tensor(v) else np.asarray(v)) for k, v in arrays.items()}
    np.savez_compressed(HERE / f"{name}.npz", **out)
    size = (HERE / f"{name}.npz").stat().st_size
    print(f"{name}.npz: {len(out)} arrays, {size / 1024:.1f} KiB")


def heat_config(nelx, nely, **kw):
    """A HeatRunConfig-shaped object carrying only the fields heat_time_field reads."""

    class Cfg:
        pass

    c = Cfg()
    c.chi_contrast = kw.get("chi_contrast", 1000.0)
    c.drain_beta = kw.get("drain_beta", 25.0)
    c.time_map = kw.get("time_map", "one_minus")
    c.heat_cg_rtol = kw.get("heat_cg_rtol", 1e-8)
    c.poisson_cg_rtol = kw.get("poisson_cg_rtol", 1e-8)
    return c


def gen_fem_basic():
    save(
        "fem_basic",
        KE=fem.plane_stress_KE(NU),
        KE_nu0=fem.plane_stress_KE(0.0),
        KEh=fem.diffusion_KE(),
        edof_5x3_d2=fem.element_dof_map(5, 3, 2),
        edof_5x3_d1=fem.element_dof_map(5, 3, 1),
        edof_7x4_d2=fem.element_dof_map(7, 4, 2),
        mbb_F=load_cases.load_case(load_cases.LoadCase.MBB, 12, 4, 0.0, 0.0, 1.0)[0],
        mbb_free=load_cases.load_case(load_cases.LoadCase.MBB, 12, 4, 0.0, 0.0, 1.0)[1],
        cant_F=load_cases.load_case(load_cases.LoadCase.CANTILEVER, 12, 4, 0.0, 0.0, 1.0)[0],
        cant_free=load_cases.load_case(load_cases.LoadCase.CANTILEVER, 12, 4, 0.0, 0.0, 1.0)[1],
        gravity_C=gravity.gravity_load_matrix(6, 4).toarray(),
        coarsen=np.array([torch_mg.coarsening_factors(a, b) for a, b in
                          [(180, 60), (45, 15), (15, 5), (5, 5), (2048, 1024), (120, 40),
                           (30, 10), (7, 9), (6, 9), (768, 384)]]),
        plate_bottom_6x4=vh.plate_nodes(6, 4, "bottom_edge"),
        plate_left_6x4=vh.plate_nodes(6, 4, "left_edge"),
    )


def gen_load_cases():
    """Every load case of the reference (load_cases.load_case, active_mask) on a few meshes
    and load / support spans, with fem.edge_load_shares and units.in_elements."""
    import sttopt.units as units

    out = {}
    for case in load_cases.LoadCase:
        for nelx, nely, load_m, sup_m, h in [(12, 8, 0.0, 0.5, 0.25), (20, 10, 0.4, 0.3, 0.1),
                                             (16, 12, 0.27, 0.13, 0.05)]:
            k = f"{case.value}_{nelx}x{nely}_{load_m}_{sup_m}_{h}"
            F, free = load_cases.load_case(case, nelx, nely, load_m, sup_m, h)
            out[f"{k}_F"], out[f"{k}_free"] = F, free
            out[f"{k}_active"] = load_cases.active_mask(case, nelx, nely)
    for n, length in [(5, 0.0), (5, 1.0), (9, 2.5), (9, 8.0), (33, 7.3)]:
        out[f"shares_{n}_{length}"] = fem.edge_load_shares(n, length)
    out["in_elements"] = np.array([units.in_elements(a, b) for a, b in [(0.3, 0.1), (1.0, 0.25), (0.35, 0.1),
                                                                        (0.7, 0.1), (1.0, 0.3)]])
    save("load_cases", **out)


def gen_operator():
    rng = np.random.default_rng(11)
    nelx, nely = 12, 8
    ndof = 2 * (nelx + 1) * (nely + 1)
    edof = t(fem.element_dof_map(nelx, nely), torch.int64)
    KE = t(fem.plane_stress_KE(NU))
    F, free = load_cases.load_case(load_cases.LoadCase.CANTILEVER, nelx, nely, 0.0, 0.0, 1.0)
    mask = torch_fem.free_mask(ndof, t(free, torch.int64))
    x = rng.uniform(0.0, 1.0, (3, nelx * nely))
    x[2, : nelx * nely // 3] = 1e-6
    dens = torch_fem.simp_density(t(x), EMIN, EMAX, PENAL)
    U = t(rng.standard_normal((3, ndof)))
    # scalar with reaction
    hx, hy = 9, 7
    hedof = t(fem.element_dof_map(hx, hy, 1), torch.int64)
    KEh = t(fem.diffusion_KE())
    hn = (hx + 1) * (hy + 1)
    hchi = t(rng.uniform(0.01, 2.0, (2, hx * hy)))
    hreac = t(rng.uniform(0.0, 0.5, (2, hx * hy)))
    hmask = ~torch.as_tensor(vh.plate_nodes(hx, hy, "bottom_edge"))
    hU = t(rng.standard_normal((2, hn)))
    rd = torch_fem.lumped_reaction(hreac, hedof, hn)
    save(
        "operator",
        x=x, U=U, mask=mask, dens=dens,
        matvec=torch_fem.matvec(U, dens, edof, KE, ndof),
        matvec_bcast=torch_fem.matvec(U, dens[0], edof, KE, ndof),
        diag=torch_fem.matvec_diagonal(dens, edof, KE, ndof),
        op=torch_fem.operator(U, dens, edof, KE, ndof, mask),
        jdiag=torch_fem.jacobi_preconditioner_diag(dens, edof, KE, ndof, mask),
        h_chi=hchi, h_reac=hreac, h_mask=hmask, h_U=hU,
        h_rdiag=rd,
        h_op=torch_fem.operator(hU, hchi, hedof, KEh, hn, hmask, rd),
        h_jdiag=torch_fem.jacobi_preconditioner_diag(hchi, hedof, KEh, hn, hmask, rd),
    )


def gen_transfers():
    rng = np.random.default_rng(12)
    out = {}
    for kx, ky in [(2, 2), (3, 3), (3, 1), (2, 3), (1, 2)]:
        for d in (1, 2):
            nCx, nCy = 3, 2
            c = t(rng.standard_normal(d * (nCx + 1) * (nCy + 1)))
            f = t(rng.standard_normal(d * (nCx * kx + 1) * (nCy * ky + 1)))
            key = f"k{kx}{ky}_d{d}"
            out[f"c_{key}"] = c
            out[f"f_{key}"] = f
            out[f"P_{key}"] = torch_mg._on_node_grid(c, nCx + 1, nCy + 1, kx, ky, torch_mg._interp_axis)
            out[f"R_{key}"] = torch_mg._on_node_grid(f, nCx * kx + 1, nCy * ky + 1, kx, ky,
                                                     torch_mg._restrict_axis)
            out[f"S_{key}"] = torch_mg.child_interpolation_matrices(kx, ky, None, F64, d)
        out[f"children_{kx}{ky}"] = torch_mg._child_elements(6 * kx, 2 * ky, kx, ky, "cpu")
    save("transfers", **out)


def _binary_design(nelx, nely):
    rows, cols = np.mgrid[0:nely, 0:nelx]
    x = np.zeros((nely, nelx))
    x[np.abs(rows / max(nely - 1, 1) - cols / max(nelx - 1, 1)) < 0.15] = 1.0
    x[:2, :] = 1.0
    x[-2:, :] = 1.0
    x[:, :2] = 1.0
    return x.ravel()


def gen_hierarchy():
    rng = np.random.default_rng(13)
    out = {}
    # vector: 24x18 (factors 2, 3) batched over 2 density rows
    nelx, nely = 24, 18
    ndof = 2 * (nelx + 1) * (nely + 1)
    F, free = load_cases.load_case(load_cases.LoadCase.CANTILEVER, nelx, nely, 0.0, 0.0, 1.0)
    mask = torch_fem.free_mask(ndof, t(free, torch.int64))
    x = np.stack([_binary_design(nelx, nely), rng.uniform(0.05, 1.0, nelx * nely)])
    dens = torch_fem.simp_density(t(x), EMIN, EMAX, PENAL)
    edof = t(fem.element_dof_map(nelx, nely), torch.int64)
    KE = t(fem.plane_stress_KE(NU))
    levels = torch_mg.build_hierarchy(dens, edof, KE, mask, nelx, nely, max_coarse_elements=10)
    out["v_x"] = x
    out["v_mask"] = mask
    out["v_nlevels"] = len(levels)
    for i, lv in enumerate(levels):
        out[f"v_L{i}_shape"] = np.array([lv.nelx, lv.nely, lv.kx, lv.ky])
        out[f"v_L{i}_diag"] = lv.diag
        out[f"v_L{i}_mask"] = lv.mask
        if lv.keff is not None:
            out[f"v_L{i}_keff"] = lv.keff
    out["v_chol"] = levels[-1].chol
    r = torch_fem.project(t(rng.standard_normal((2, ndof))), mask)
    M = torch_mg.VCycle(levels)
    out["v_r"] = r
    out["v_Mr"] = M(r)
    out["v_Ar"] = levels[0](r)
    # scalar with reaction, 18x12
    hx, hy = 18, 12
    hn = (hx + 1) * (hy + 1)
    hedof = t(fem.element_dof_map(hx, hy, 1), torch.int64)
    KEh = t(fem.diffusion_KE())
    hmask = ~torch.as_tensor(vh.plate_nodes(hx, hy, "bottom_edge"))
    hchi = t(rng.uniform(1e-3, 1.0, hx * hy))
    hreac = torch.full((hx * hy,), 25.0 / (hx * hy), dtype=F64)
    hl = torch_mg.build_hierarchy(hchi, hedof, KEh, hmask, hx, hy, reaction=hreac,
                                  max_coarse_elements=10)
    out["h_chi"] = hchi
    out["h_nlevels"] = len(hl)
    for i, lv in enumerate(hl):
        out[f"h_L{i}_shape"] = np.array([lv.nelx, lv.nely, lv.kx, lv.ky])
        out[f"h_L{i}_diag"] = lv.diag
        out[f"h_L{i}_mask"] = lv.mask
        if lv.keff is not None:
            out[f"h_L{i}_keff"] = lv.keff
    out["h_chol"] = hl[-1].chol
    hr = torch_fem.project(t(rng.standard_normal(hn)), hmask)
    out["h_r"] = hr
    out["h_Mr"] = torch_mg.VCycle(hl)(hr)
    save("hierarchy", **out)


def gen_mbb_config():
    """MBB 120x40, uniform 0.5, one MG-PCG solve, compliance and dc/dxPhys."""
    nelx, nely = 120, 40
    F, free = load_cases.load_case(load_cases.LoadCase.MBB, nelx, nely, 0.0, 0.0, 1.0)
    ndof = len(F)
    KE = t(fem.plane_stress_KE(NU))
    edof = t(fem.element_dof_map(nelx, nely), torch.int64)
    mask = torch_fem.free_mask(ndof, t(free, torch.int64))
    xPhys = torch.full((nely, nelx), 0.5, dtype=F64, requires_grad=True)
    info = {}
    density = torch_fem.simp_density(xPhys, EMIN, EMAX, PENAL).flatten()
    U = torch_solve.femsolve(density, t(F), edof, KE, mask, nelx, nely, info=info)
    ce = compliance._element_strain_energy(U, edof, KE, nely, nelx)
    c = torch.sum(torch_fem.simp_density(xPhys, EMIN, EMAX, PENAL) * ce)
    (dc,) = sensitivity.jacobian_rows(c[None], [xPhys])
    levels = torch_mg.build_hierarchy(density.detach(), edof, KE, mask, nelx, nely)
    save("mbb120x40", F=F, mask=mask, U=U, c=c, dc=dc.reshape(nely, nelx),
         forward_n_iter=info["forward_n_iter"], backward_n_iter=info["backward_n_iter"],
         level_shapes=np.array([[lv.nelx, lv.nely] for lv in levels]),
         coarse_ndof=levels[-1].ndof)


def gen_cantilever():
    """Config-2 shape, reduced: mid-right load cantilever, smoothed density, FP64."""
    out = {}
    for nelx, nely, seed, mce in [(64, 32, 2, 700), (96, 48, 3, 60)]:
        x = smoothed_density(nelx, nely, seed)
        nodes = fem.node_grid(nelx, nely)
        ndof = 2 * nodes.size
        F = np.zeros(ndof)
        F[2 * nodes[nely // 2, -1] + 1] = -1.0
        mask = np.ones(ndof, bool)
        mask[2 * nodes[:, 0]] = False
        mask[2 * nodes[:, 0] + 1] = False
        KE = t(fem.plane_stress_KE(NU))
        edof = t(fem.element_dof_map(nelx, nely), torch.int64)
        xPhys = t(x).requires_grad_(True)
        info = {}
        density = torch_fem.simp_density(xPhys, EMIN, EMAX, PENAL).flatten()
        U = torch_solve.femsolve(density, t(F), edof, KE, torch.as_tensor(mask), nelx, nely,
                                 info=info, max_coarse_elements=mce)
        ce = compliance._element_strain_energy(U, edof, KE, nely, nelx)
        c = torch.sum(torch_fem.simp_density(xPhys, EMIN, EMAX, PENAL) * ce)
        (dc,) = sensitivity.jacobian_rows(c[None], [xPhys])
        k = f"{nelx}x{nely}"
        out.update({f"{k}_x": x, f"{k}_F": F, f"{k}_mask": mask, f"{k}_U": U, f"{k}_c": c,
                    f"{k}_dc": dc.reshape(nely, nelx), f"{k}_mce": mce,
                    f"{k}_fwd_iter": info["forward_n_iter"], f"{k}_bwd_iter": info["backward_n_iter"]})
    save("cantilever", **out)


def _heat(nelx, nely, x, mu, w, conduction_penal=3.0, mce=700):
    mesh = vh.ScalarMesh.build(nelx, nely, "bottom_edge", torch.device("cpu"), F64)
    cfg = heat_config(nelx, nely)
    xPhys = t(x).requires_grad_(True)
    muT = t(mu).requires_grad_(True)
    orig = torch_mg.MAX_COARSE_ELEMENTS
    sol = vh.heat_time_field(cfg, mesh, xPhys, muT, conduction_penal=conduction_penal)
    J = torch.sum(t(w) * sol.tPhys)
    gx, gmu = torch.autograd.grad(J, [xPhys, muT])
    return sol, J, gx, gmu


def gen_heat():
    out = {}
    for nelx, nely, seed in [(40, 20, 4), (60, 30, 5)]:
        rng = np.random.default_rng(seed)
        x = smoothed_density(nelx, nely, seed)
        mu = rng.uniform(0.2, 0.8, (nely, nelx))
        w = rng.uniform(-1, 1, (nely, nelx))
        sol, J, gx, gmu = _heat(nelx, nely, x, mu, w)
        k = f"{nelx}x{nely}"
        out.update({f"{k}_x": x, f"{k}_mu": mu, f"{k}_w": w, f"{k}_tPhys": sol.tPhys,
                    f"{k}_T": sol.primary, f"{k}_J": J, f"{k}_gx": gx, f"{k}_gmu": gmu})
    save("heat", **out)


def _hard_time_mask(tPhys, ti, beta):
    return (tPhys <= ti).to(tPhys.dtype)


def spacetime_reference(x, w, n_stage, rtol=1e-8):
    """The space-time objective of the configs, composed from reference functions.

    ``compliance.time_mask`` is replaced by the hard threshold ``tPhys <= s/n_stage``;
    the stage rows go through one batched ``femsolve`` exactly as
    ``batched_whole_and_gravity_compliance`` stacks them (without its row 0).  ``rtol``
    is the heat solve's and the stage solves' (and their adjoints') tolerance.
    """
    nely, nelx = x.shape
    mesh = vh.ScalarMesh.build(nelx, nely, "bottom_edge", torch.device("cpu"), F64)
    cfg = heat_config(nelx, nely, heat_cg_rtol=rtol)
    xPhys = t(x).requires_grad_(True)
    mu = torch.full((nely, nelx), 0.5, dtype=F64)
    sol = vh.heat_time_field(cfg, mesh, xPhys, mu, conduction_penal=3.0)
    tPhys = sol.tPhys
    ndof = 2 * (nelx + 1) * (nely + 1)
    KE = t(fem.plane_stress_KE(NU))
    edof = t(fem.element_dof_map(nelx, nely), torch.int64)
    nodes = fem.node_grid(nelx, nely)
    mask = np.ones(ndof, bool)
    mask[2 * nodes[-1, :]] = False
    mask[2 * nodes[-1, :] + 1] = False
    mask = torch.as_tensor(mask)
    C = torch_util.csr_to_tensor(gravity.gravity_load_matrix(nelx, nely), "cpu", F64)
    orig = compliance.time_mask
    compliance.time_mask = _hard_time_mask
    try:
        rows, Fs, xts = [], [], []
        for s in range(1, n_stage + 1):
            _, xt, Fg = compliance._gravity_load(xPhys, tPhys, s / n_stage, C, 10.0, ndof)
            rows.append(torch_fem.simp_density(xt, EMIN, EMAX, PENAL).flatten())
            Fs.append(Fg)
            xts.append(xt)
    finally:
        compliance.time_mask = orig
    density = torch.stack(rows)
    info = {}
    U = torch_solve.femsolve(density, torch.stack(Fs), edof, KE, mask, nelx, nely, info=info, rtol=rtol)
    cs = []
    for i, xt in enumerate(xts):
        ce = compliance._element_strain_energy(U[i], edof, KE, nely, nelx)
        cs.append(torch.sum(torch_fem.simp_density(xt, EMIN, EMAX, PENAL) * ce))
    cs = torch.stack(cs)
    Jt = torch.sum(t(w) * tPhys)
    L = cs.sum() + Jt
    (g,) = sensitivity.jacobian_rows(L[None], [xPhys])
    member = np.stack([(tPhys.detach().numpy().ravel() <= s / n_stage) for s in range(1, n_stage + 1)])
    return dict(x=x, w=w, tPhys=tPhys, T=sol.primary, U=U, c_s=cs, J_t=Jt, L=L,
                grad=g.reshape(nely, nelx), member=member.astype(np.uint8),
                fwd_iter=info["forward_n_iter"], bwd_iter=info["backward_n_iter"])


def gen_spacetime():
    out = {}
    for nelx, nely, n_stage, seed in [(48, 24, 4, 7), (64, 32, 16, 8)]:
        rng = np.random.default_rng(seed)
        x = smoothed_density(nelx, nely, seed)
        w = rng.uniform(-1, 1, (nely, nelx))
        res = spacetime_reference(x, w, n_stage)
        k = f"{nelx}x{nely}s{n_stage}"
        out.update({f"{k}_{name}": v for name, v in res.items()})
    save("spacetime", **out)


def gen_spacetime_512():
    """The differentiation configuration: the space-time objective at 512x256, 16 stages.

    Inputs are regenerated from the seed by the tests (``smoothed_density`` and
    ``default_rng(seed).uniform``); only their checksums are stored, with the reference's
    outputs (stage membership bit-packed)."""
    nelx, nely, n_stage, seed = 512, 256, 16, 4
    rng = np.random.default_rng(seed)
    x = smoothed_density(nelx, nely, seed)
    w = rng.uniform(-1, 1, (nely, nelx))
    res = spacetime_reference(x, w, n_stage)
    save("spacetime512", x_sum=x.sum(), w_sum=w.sum(), tPhys=res["tPhys"], c_s=res["c_s"],
         J_t=res["J_t"], L=res["L"], grad=res["grad"], member_bits=np.packbits(res["member"], axis=-1),
         fwd_iter=res["fwd_iter"], bwd_iter=res["bwd_iter"])


def gen_cantilever_full():
    """Config 2 at its size: the 1024x512 cantilever (left edge clamped, unit -y load at the
    mid-right node), seeded radius-4 smoothed density in [1e-3, 1], FP64, the reference's
    6-level hierarchy; U, c and dc/dxPhys at the config's rtol 1e-8 (iteration counts) and
    at rtol 1e-12 (values with the solve noise removed).  Inputs are regenerated by the
    tests from the seed; fields are stored as summaries."""
    nelx, nely, seed = 1024, 512, 2
    x = smoothed_density(nelx, nely, seed)
    nodes = fem.node_grid(nelx, nely)
    ndof = 2 * nodes.size
    F = np.zeros(ndof)
    F[2 * nodes[nely // 2, -1] + 1] = -1.0
    mask = np.ones(ndof, bool)
    mask[2 * nodes[:, 0]] = False
    mask[2 * nodes[:, 0] + 1] = False
    KE = t(fem.plane_stress_KE(NU))
    edof = t(fem.element_dof_map(nelx, nely), torch.int64)
    out = {"x_sum": x.sum(), "nelx": nelx, "nely": nely, "seed": seed}
    for tag, rtol in (("r8", 1e-8), ("r12", 1e-12)):
        xPhys = t(x).requires_grad_(True)
        info = {}
        density = torch_fem.simp_density(xPhys, EMIN, EMAX, PENAL).flatten()
        U = torch_solve.femsolve(density, t(F), edof, KE, torch.as_tensor(mask), nelx, nely, info=info, rtol=rtol)
        ce = compliance._element_strain_energy(U, edof, KE, nely, nelx)
        c = torch.sum(torch_fem.simp_density(xPhys, EMIN, EMAX, PENAL) * ce)
        (dc,) = sensitivity.jacobian_rows(c[None], [xPhys])
        out.update({f"{tag}_c": c.detach(), f"{tag}_fwd_iter": info["forward_n_iter"],
                    f"{tag}_bwd_iter": info["backward_n_iter"]})
        out.update(field_summary(f"{tag}_U", U.detach().numpy(), 101, 97))
        out.update(field_summary(f"{tag}_dc", dc.numpy(), 102, 61))
    levels = torch_mg.build_hierarchy(torch_fem.simp_density(t(x), EMIN, EMAX, PENAL).flatten(), edof, KE,
                                      torch.as_tensor(mask), nelx, nely)
    out["level_shapes"] = np.array([[lv.nelx, lv.nely] for lv in levels])
    out["coarse_ndof"] = levels[-1].ndof
    save("cantilever1024", **out)


def _member_hash(member):
    """Per stage: the member count and two index sums (int64, exact), pinning the stage
    membership of millions of elements in three integers a stage."""
    m = np.asarray(member, dtype=bool)
    idx = np.arange(m.shape[-1], dtype=np.int64)
    return np.stack([m.sum(-1), (m * idx).sum(-1), (m * (idx * idx % 1000003)).sum(-1)], axis=1)


def gen_spacetime_full(nelx, nely, seed, rtols=(1e-8, 1e-12)):
    """The space-time objective of the configs at a benchmark size, 16 stages: the
    reference's heat solve, hard-threshold stages, one batched stage femsolve and the
    sensitivity field, at each ``rtol``.  ``seed`` gives the density (``smoothed_density``)
    and the time weights (``default_rng(seed).uniform(-1, 1)``), the benchmark's recipe."""
    import time

    n_stage = 16
    x = smoothed_density(nelx, nely, seed)
    w = np.random.default_rng(seed).uniform(-1, 1, (nely, nelx))
    out = {"x_sum": x.sum(), "w_sum": w.sum(), "nelx": nelx, "nely": nely, "seed": seed, "n_stage": n_stage}
    for rtol in rtols:
        tag = f"r{round(-np.log10(rtol))}"
        t0 = time.perf_counter()
        res = spacetime_reference(x, w, n_stage, rtol=rtol)
        print(f"  spacetime {nelx}x{nely} rtol {rtol:g}: {time.perf_counter() - t0:.1f} s", flush=True)
        U = res["U"].detach().numpy()
        out.update({f"{tag}_c_s": res["c_s"].detach(), f"{tag}_J_t": res["J_t"].detach(),
                    f"{tag}_L": res["L"].detach(), f"{tag}_fwd_iter": res["fwd_iter"],
                    f"{tag}_bwd_iter": res["bwd_iter"], f"{tag}_member": _member_hash(res["member"]),
                    f"{tag}_U_norms": np.linalg.norm(U, axis=1)})
        out.update(field_summary(f"{tag}_grad", res["grad"].numpy(), 201, 257))
        out.update(field_summary(f"{tag}_tPhys", res["tPhys"].detach().numpy(), 202, 263))
        out.update(field_summary(f"{tag}_U", U, 203, 4099))
        del res, U
    save(f"spacetime{nelx}", **out)


def gen_filters():
    """The cone density filter and the Heaviside projection, as the reference computes
    them (filters.density_filter / apply_density_filter / heaviside_projection*), and the
    gradient of sum(w * P(H x / Hs)) through the reference's autograd (symmetric_matmul)."""
    out = {}
    for nelx, nely, rmin, seed in [(37, 23, 1.5, 11), (37, 23, 2.5, 12), (64, 40, 4.0, 13), (20, 11, 8.0, 14)]:
        k = f"{nelx}x{nely}r{rmin}"
        H, Hs = filters.density_filter(nelx, nely, rmin)
        rng = np.random.default_rng(seed)
        x = rng.uniform(0, 1, (nely, nelx))
        w = rng.uniform(-1, 1, (nely, nelx))
        Ht = torch_util.symmetric_csr_to_tensor(H, "cpu", F64)
        xt_t = t(x).requires_grad_(True)
        xTilde = filters.apply_density_filter(xt_t, Ht, t(Hs))
        out[f"{k}_x"], out[f"{k}_w"], out[f"{k}_Hs"] = x, w, Hs
        out[f"{k}_xTilde"] = xTilde.detach().numpy()
        for beta in (1.0, 8.0, float("inf")):
            xp = filters.heaviside_projection(xTilde, beta, 0.5)
            out[f"{k}_b{beta}_xPhys"] = xp.detach().numpy()
            if not np.isinf(beta):
                out[f"{k}_b{beta}_dP"] = filters.heaviside_projection_derivative(xTilde, beta, 0.5).detach().numpy()
                (g,) = torch.autograd.grad(torch.sum(t(w) * xp), [xt_t], retain_graph=True)
                out[f"{k}_b{beta}_grad"] = g.numpy()
        (g,) = torch.autograd.grad(torch.sum(t(w) * xTilde), [xt_t])
        out[f"{k}_grad_filter"] = g.numpy()
    save("filters", **out)


def gen_compliance_smooth():
    """The production stage glue with the smooth stage mask: batched_whole_and_gravity_compliance
    (row 0 = the point-load whole structure, then one self-weight row per stage time) on an MBB
    grid, and the gradient of c + sum_s w_s c_s in xPhys and tPhys through the reference's
    autograd (its dcx and dct)."""
    out = {}
    for nelx, nely, beta_t, times, seed in [(48, 24, 10.0, (0.25, 0.5, 0.75, 1.0), 21),
                                            (40, 16, 40.0, (0.2, 0.45, 0.7), 22)]:
        k = f"{nelx}x{nely}"
        ndof = 2 * (nelx + 1) * (nely + 1)
        # the MBB point load on the whole-structure row; the build plate (the bottom row of
        # nodes, both dofs) clamped, as the space-time stages are supported
        F, _ = load_cases.load_case(load_cases.LoadCase.MBB, nelx, nely, 0.0, 0.0, 1.0)
        plate = fem.node_grid(nelx, nely)[-1, :]
        free = np.setdiff1d(np.arange(ndof), np.concatenate([2 * plate, 2 * plate + 1]))
        rng = np.random.default_rng(seed)
        x = smoothed_density(nelx, nely, seed)
        # a layered build from the bottom (the supports' side) with a mild seeded ripple,
        # so every stage's material is connected to the supports
        rows = (nely - 0.5 - np.arange(nely)[:, None]) / nely
        tp = np.clip(rows + 0.05 * np.sin(0.3 * np.arange(nelx))[None, :] + 0.02 * rng.uniform(-1, 1, (nely, nelx)),
                     0.0, 1.0)
        w = rng.uniform(0.5, 1.5, len(times))
        C = torch_util.csr_to_tensor(gravity.gravity_load_matrix(nelx, nely), "cpu", F64)
        xT, tT = t(x).requires_grad_(True), t(tp).requires_grad_(True)
        c, stages, U = compliance.batched_whole_and_gravity_compliance(
            xT, tT, t(fem.plane_stress_KE(NU)), t(fem.element_dof_map(nelx, nely), torch.int64), EMIN, EMAX,
            PENAL, t(free, torch.int64), t(F), ndof, C, beta_t, list(times))
        L = c + sum(float(wi) * cs for wi, cs in zip(w, stages))
        gx, gt = torch.autograd.grad(L, [xT, tT])
        out.update({f"{k}_x": x, f"{k}_t": tp, f"{k}_w": w, f"{k}_beta_t": beta_t, f"{k}_times": np.array(times),
                    f"{k}_F": F, f"{k}_free": free, f"{k}_c": c, f"{k}_stages": torch.stack(stages), f"{k}_U": U,
                    f"{k}_L": L, f"{k}_gx": gx, f"{k}_gt": gt})
    out["C_7x4"] = gravity.gravity_load_matrix(7, 4).toarray()
    save("compliance_smooth", **out)


def gen_compliance_single():
    """The single-solve glue (whole_compliance, gravity_compliance, _gravity_load) with its
    autograd gradients, and the batched call with the stage mask replaced by the hard
    threshold (the space-time configurations' membership), on one MBB-loaded grid with the
    build plate clamped."""
    nelx, nely, seed = 36, 20, 23
    ndof = 2 * (nelx + 1) * (nely + 1)
    F, _ = load_cases.load_case(load_cases.LoadCase.MBB, nelx, nely, 0.0, 0.0, 1.0)
    plate = fem.node_grid(nelx, nely)[-1, :]
    free = np.setdiff1d(np.arange(ndof), np.concatenate([2 * plate, 2 * plate + 1]))
    rng = np.random.default_rng(seed)
    x = smoothed_density(nelx, nely, seed)
    rows = (nely - 0.5 - np.arange(nely)[:, None]) / nely
    tp = np.clip(rows + 0.03 * rng.uniform(-1, 1, (nely, nelx)), 0.0, 1.0)
    wF = rng.normal(size=ndof)
    wx = rng.normal(size=(nely, nelx))
    KE = t(fem.plane_stress_KE(NU))
    edof = t(fem.element_dof_map(nelx, nely), torch.int64)
    C = torch_util.csr_to_tensor(gravity.gravity_load_matrix(nelx, nely), "cpu", F64)
    out = {"x": x, "t": tp, "F": F, "free": free, "wF": wF, "wx": wx, "rtol": 1e-12}

    # every solve at rtol 1e-12, through the reference's documented patch points (one of
    # the stages is a nearly disconnected build, whose compliance an rtol-1e-8 solve
    # fixes only to ~1e-8)
    def solve_fe(KE_, xPhys, Emin, Emax, penal, edofMat, freedofs, F_, ndof_, *, x0=None):
        nely_, nelx_ = xPhys.shape
        density = torch_fem.simp_density(xPhys, Emin, Emax, penal)
        m = torch_fem.free_mask(ndof_, freedofs, device=xPhys.device)
        return torch_solve.femsolve(density.flatten(), F_, edofMat, KE_, m, nelx_, nely_, x0=x0, rtol=1e-12)

    def solve_fe_batched(KE_, density, edofMat, m, nelx_, nely_, F_, *, x0=None):
        return torch_solve.femsolve(density, F_, edofMat, KE_, m, nelx_, nely_, x0=x0, rtol=1e-12)

    saved = compliance._solve_fe, compliance._solve_fe_batched
    compliance._solve_fe, compliance._solve_fe_batched = solve_fe, solve_fe_batched
    try:
        _compliance_single_cases(out, x, tp, F, free, wF, wx, KE, edof, C, ndof)
    finally:
        compliance._solve_fe, compliance._solve_fe_batched = saved
    save("compliance_single", **out)


def _compliance_single_cases(out, x, tp, F, free, wF, wx, KE, edof, C, ndof):
    xT = t(x).requires_grad_(True)
    c, U = compliance.whole_compliance(xT, KE, edof, EMIN, EMAX, PENAL, t(free, torch.int64), t(F), ndof)
    (gx,) = torch.autograd.grad(c, [xT])
    out.update(whole_c=c, whole_U=U, whole_gx=gx)
    xT, tT = t(x).requires_grad_(True), t(tp).requires_grad_(True)
    cg, Ug = compliance.gravity_compliance(xT, tT, KE, edof, EMIN, EMAX, PENAL, 0.55, C, 12.0,
                                           t(free, torch.int64), ndof)
    gx, gt = torch.autograd.grad(cg, [xT, tT])
    out.update(grav_c=cg, grav_U=Ug, grav_gx=gx, grav_gt=gt)
    xT, tT = t(x).requires_grad_(True), t(tp).requires_grad_(True)
    tm, xj, Fg = compliance._gravity_load(xT, tT, 0.4, C, 8.0, ndof)
    J = torch.sum(t(wF) * Fg) + torch.sum(t(wx) * xj)
    gx, gt = torch.autograd.grad(J, [xT, tT])
    out.update(gl_mask=tm, gl_xt=xj, gl_F=Fg, gl_gx=gx, gl_gt=gt)
    orig = compliance.time_mask
    compliance.time_mask = _hard_time_mask
    try:
        xT = t(x).requires_grad_(True)
        c, stages, U = compliance.batched_whole_and_gravity_compliance(
            xT, t(tp), KE, edof, EMIN, EMAX, PENAL, t(free, torch.int64), t(F), ndof, C, 10.0, [0.3, 0.6, 1.0])
        (gx,) = torch.autograd.grad(c + 2.0 * stages[0] + stages[1] + 0.5 * stages[2], [xT])
    finally:
        compliance.time_mask = orig
    out.update(hard_c=c, hard_stages=torch.stack(stages), hard_U=U, hard_gx=gx)


def laplace_config(time_map):
    """A LaplaceRunConfig-shaped object carrying only the fields laplace_time_field reads."""

    class Cfg:
        pass

    c = Cfg()
    c.chi_contrast = 100.0
    c.chi_density_floor = 1e-2
    c.chi_density_sensitivity = True
    c.laplace_cg_rtol = 1e-10
    c.poisson_cg_rtol = 1e-10
    c.time_map = time_map
    return c


def gen_time_maps():
    """The poisson map of heat_time_field and laplace_time_field (identity and poisson maps)
    with the reference's autograd gradients of sum(w tPhys); and the fused Poisson load
    divergence_load(w, direction_field(s)) with its vector-Jacobian products."""
    out = {}
    nelx, nely, seed = 40, 20, 31
    rng = np.random.default_rng(seed)
    x = smoothed_density(nelx, nely, seed)
    mu = rng.uniform(0.2, 0.8, (nely, nelx))
    w = rng.uniform(-1, 1, (nely, nelx))
    mesh = vh.ScalarMesh.build(nelx, nely, "bottom_edge", torch.device("cpu"), F64)
    cfg = heat_config(nelx, nely, time_map="poisson", heat_cg_rtol=1e-10, poisson_cg_rtol=1e-10)
    xT, muT = t(x).requires_grad_(True), t(mu).requires_grad_(True)
    sol = vh.heat_time_field(cfg, mesh, xT, muT, conduction_penal=3.0)
    J = torch.sum(t(w) * sol.tPhys)
    gx, gmu = torch.autograd.grad(J, [xT, muT])
    out.update({"heat_x": x, "heat_mu": mu, "heat_w": w, "heat_tPhys": sol.tPhys, "heat_T": sol.primary,
                "heat_phi": sol.poisson, "heat_J": J, "heat_gx": gx, "heat_gmu": gmu})

    # Poisson load alone, on a random field, with random output weights
    s_field = rng.normal(size=mesh.ndof)
    we = rng.uniform(0.1, 1.0, nelx * nely)
    gF = rng.normal(size=mesh.ndof)
    sT, weT = t(s_field).requires_grad_(True), t(we).requires_grad_(True)
    Fp = mesh.divergence_load(weT, mesh.direction_field(sT))
    gs, gw = torch.autograd.grad(torch.sum(t(gF) * Fp), [sT, weT])
    u = rng.normal(size=(2, mesh.ndof))
    out.update({"pl_s": s_field, "pl_w": we, "pl_gF": gF, "pl_F": Fp, "pl_gs": gs, "pl_gw": gw,
                "em_u": u, "em_means": vh.element_means(t(u), mesh.edof)})

    for nelx, nely, base, tmap, dexp, seed in [(36, 18, "bottom_edge", "identity", 0.0, 32),
                                              (36, 18, "left_edge", "identity", 1.0, 33),
                                              (32, 16, "bottom_edge", "poisson", 1.0, 34)]:
        k = f"lap_{nelx}x{nely}_{base}_{tmap}_{dexp}"
        rng = np.random.default_rng(seed)
        x = smoothed_density(nelx, nely, seed)
        mu = rng.uniform(0.2, 0.8, (nely, nelx))
        w = rng.uniform(-1, 1, (nely, nelx))
        mesh = vh.ScalarMesh.build(nelx, nely, base, torch.device("cpu"), F64)
        n_arc = mesh.arc.numel()
        b = 0.5 * np.sin(np.linspace(0.1, 3.0, n_arc)) + 0.6 + 0.05 * rng.uniform(size=n_arc)
        xT, muT, bT = t(x).requires_grad_(True), t(mu).requires_grad_(True), t(b).requires_grad_(True)
        sol = vh.laplace_time_field(laplace_config(tmap), mesh, xT, muT, bT, density_exponent=dexp)
        J = torch.sum(t(w) * sol.tPhys)
        grads = torch.autograd.grad(J, [xT, muT, bT], allow_unused=True)
        gx, gmu, gb = [torch.zeros(1, dtype=F64) if g is None else g for g in grads]
        out.update({f"{k}_x": x, f"{k}_mu": mu, f"{k}_w": w, f"{k}_b": b, f"{k}_arc": mesh.arc,
                    f"{k}_tPhys": sol.tPhys, f"{k}_u": sol.primary, f"{k}_J": J, f"{k}_gx": gx,
                    f"{k}_gmu": gmu, f"{k}_gb": gb})
        if sol.poisson is not None:
            out[f"{k}_phi"] = sol.poisson
    # wall arcs: every plate side, and an L-shaped domain (a re-entrant corner)
    lshape = np.ones((8, 12), bool)
    lshape[:4, 6:] = False
    for base in ("bottom_edge", "left_edge", "right_edge"):
        out[f"arc_rect_{base}"] = vh.wall_arc(13, 7, base)
        out[f"arc_L_{base}"] = vh.wall_arc(12, 8, base, lshape)
        out[f"plate_L_{base}"] = vh.plate_nodes(12, 8, base, lshape)
    out["lshape"] = lshape
    # the Laplace loop's wall design helpers and the start check
    for n_arc, rmin in [(30, 1.0), (30, 3.5), (45, 6.0), (5, 8.0)]:
        out[f"wf_{n_arc}_{rmin}"] = vh.wall_filter(n_arc, rmin)
    for key, (nx, ny, base, act) in {"rect": (13, 7, "bottom_edge", None), "L": (12, 8, "left_edge", lshape),
                                     "Lb": (12, 8, "bottom_edge", lshape)}.items():
        mesh = vh.ScalarMesh.build(nx, ny, base, torch.device("cpu"), F64, act)
        out[f"dw_{key}"] = vh.distance_wall(mesh)
    rng = np.random.default_rng(41)
    mesh = vh.ScalarMesh.build(10, 6, "bottom_edge", torch.device("cpu"), F64)
    t_nodes = rng.uniform(-0.05, 1.0, mesh.ndof)
    t_el = rng.uniform(0.0, 1.0, (6, 10))
    solid = rng.uniform(size=(6, 10)) > 0.4
    base_el = np.arange(50, 60)
    sol = vh.TimeFieldSolution(t(t_el), t(t_nodes), None, t(t_nodes))
    rep = vh.start_report(mesh, sol, solid, base_el)
    out.update({"sr_t": t_nodes, "sr_tPhys": t_el, "sr_solid": solid, "sr_base": base_el,
                "sr_report": np.array(repr(sorted(rep.items())))})
    save("time_maps", **out)


def gen_neg_log():
    """``heat_time_field`` with the ``neg_log`` map (t = -log(max(T, 0) + floor), the floor
    a fraction of the smallest element mean of T over the part) and the reference's
    autograd gradients of sum(w tPhys) in xPhys and mu; solves at rtol 1e-10."""
    out = {}
    for nelx, nely, seed in [(40, 20, 51), (64, 24, 52)]:
        rng = np.random.default_rng(seed)
        x = smoothed_density(nelx, nely, seed)
        mu = rng.uniform(0.2, 0.8, (nely, nelx))
        w = rng.uniform(-1, 1, (nely, nelx))
        mesh = vh.ScalarMesh.build(nelx, nely, "bottom_edge", torch.device("cpu"), F64)
        cfg = heat_config(nelx, nely, time_map="neg_log", heat_cg_rtol=1e-10)
        xT, muT = t(x).requires_grad_(True), t(mu).requires_grad_(True)
        sol = vh.heat_time_field(cfg, mesh, xT, muT, conduction_penal=3.0)
        J = torch.sum(t(w) * sol.tPhys)
        gx, gmu = torch.autograd.grad(J, [xT, muT])
        k = f"{nelx}x{nely}"
        out.update({f"{k}_x": x, f"{k}_mu": mu, f"{k}_w": w, f"{k}_tPhys": sol.tPhys, f"{k}_T": sol.primary,
                    f"{k}_t_nodes": sol.t, f"{k}_J": J, f"{k}_gx": gx, f"{k}_gmu": gmu})
    save("neg_log", **out)


def gen_pcg_cases():
    """Retirement, zero rows, warm starts and non-convergence, as the reference does them."""
    nelx, nely = 18, 12
    ndof = 2 * (nelx + 1) * (nely + 1)
    F, free = load_cases.load_case(load_cases.LoadCase.CANTILEVER, nelx, nely, 0.0, 0.0, 1.0)
    mask = torch_fem.free_mask(ndof, t(free, torch.int64))
    KE = t(fem.plane_stress_KE(NU))
    edof = t(fem.element_dof_map(nelx, nely), torch.int64)
    x = np.stack([_binary_design(nelx, nely), np.full(nelx * nely, 0.4), np.full(nelx * nely, 0.9)])
    Fb = t(F).expand(3, -1).clone()
    Fb[1] = 0.0
    info = {}
    U, n = torch_mg.solve(Fb, t(x), edof, KE, EMIN, EMAX, PENAL, mask, nelx, nely,
                          rtol=1e-11, max_coarse_elements=24, info=info)
    try:
        torch_mg.solve(Fb, t(x), edof, KE, EMIN, EMAX, PENAL, mask, nelx, nely,
                       rtol=1e-14, max_iter=2, max_coarse_elements=24)
        raise AssertionError("expected non-convergence")
    except torch_fem.CGConvergenceError as e:
        resid = e.residuals
        msg = str(e)
    save("pcg_cases", x=x, F=Fb, mask=mask, U=U, n_iter=n, row_iters=info["row_iters"],
         fail_resid=resid, fail_msg=np.array(msg))


def _mma_problem(rng, m, n, iteration):
    """A seeded MMA subproblem of the shape the optimisation loop builds: variables in
    [0, 1] away from the bounds, gradients of both signs, some constraints violated."""
    xmin, xmax = np.zeros(n), np.ones(n)
    xval = rng.uniform(0.05, 0.95, n)
    xold1 = np.clip(xval + rng.normal(0, 0.02, n), 0.0, 1.0)
    xold2 = np.clip(xold1 + rng.normal(0, 0.02, n), 0.0, 1.0)
    low = xval - rng.uniform(0.1, 0.4, n)
    upp = xval + rng.uniform(0.1, 0.4, n)
    return dict(m=m, n=n, iteration=iteration, xval=xval, xmin=xmin, xmax=xmax, xold1=xold1, xold2=xold2,
                f0val=float(rng.normal()), df0dx=rng.normal(0, 1.0, n), fval=rng.normal(0, 0.5, m),
                dfdx=rng.normal(0, 1.0, (m, n)), low=low, upp=upp, a0=1.0, a=np.zeros(m),
                c=np.full(m, 1000.0), d=rng.uniform(0.0, 1.0, m))


def gen_mma():
    """``mma.mmasub`` (asymptotes, the separable approximation and ``subsolv``'s
    primal-dual Newton solve) on seeded subproblems: the first-iteration asymptotes
    (m = 1), the adaptive branch with per-variable trust regions from
    ``trust_region_params`` (m = 3), more constraints (m = 12), and the m >= n
    elimination (m = 6, n = 4)."""
    import sttopt.mma as mma

    rng = np.random.default_rng(11)
    cases = [("first", 1, 2000, 0, None), ("adapt", 3, 5000, 5, "trust"), ("wide", 12, 3000, 3, None),
             ("mgen", 6, 4, 4, None)]
    out = {}
    names = ("xmma", "ymma", "zmma", "lam", "xsi", "eta", "mu", "zet", "s", "low", "upp")
    for tag, m, n, it, kind in cases:
        p = _mma_problem(rng, m, n, it)
        kw = {}
        if kind == "trust":
            tr = mma.trust_region_params(t(rng.uniform(0.02, 0.1, n)), t(p["xmax"] - p["xmin"]))
            kw = dict(tr)
            for k, v in tr.items():
                out[f"{tag}_{k}"] = v.numpy()
        res = mma.mmasub(m, n, it, t(p["xval"]), t(p["xmin"]), t(p["xmax"]), t(p["xold1"]), t(p["xold2"]),
                         p["f0val"], t(p["df0dx"]), t(p["fval"]), t(p["dfdx"]), t(p["low"]), t(p["upp"]), p["a0"],
                         t(p["a"]), t(p["c"]), t(p["d"]), **kw)
        for k, v in p.items():
            out[f"{tag}_in_{k}"] = np.asarray(v)
        for k, v in zip(names, res):
            out[f"{tag}_{k}"] = np.asarray(v.detach().cpu().numpy() if torch.is_tensor(v) else v)
    save("mma", **out)


GENERATORS = {
    "fem_basic": gen_fem_basic, "load_cases": gen_load_cases, "operator": gen_operator, "transfers": gen_transfers,
    "hierarchy": gen_hierarchy, "pcg_cases": gen_pcg_cases, "mbb120x40": gen_mbb_config,
    "cantilever": gen_cantilever, "heat": gen_heat, "spacetime": gen_spacetime, "filters": gen_filters,
    "compliance_smooth": gen_compliance_smooth, "compliance_single": gen_compliance_single,
    "time_maps": gen_time_maps, "neg_log": gen_neg_log, "mma": gen_mma,
}
OPTIONAL = {
    "spacetime512": gen_spacetime_512,
    "cantilever1024": gen_cantilever_full,
    "spacetime1024": lambda: gen_spacetime_full(1024, 512, 5),
    "spacetime2048": lambda: gen_spacetime_full(2048, 1024, 3),
}


if __name__ == "__main__":
    torch.set_num_threads(os.cpu_count() or 1)
    if "--only" in sys.argv:
        names = sys.argv[sys.argv.index("--only") + 1].split(",")
    else:
        names = list(GENERATORS)
        if "--with-512" in sys.argv:
            names.append("spacetime512")
        if "--full-size" in sys.argv:
            names += ["cantilever1024", "spacetime1024", "spacetime2048"]
    for name in names:
        (GENERATORS.get(name) or OPTIONAL[name])()
