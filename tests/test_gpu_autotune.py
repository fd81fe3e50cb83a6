"""The launch-shape autotuner (``sttopt_b200.autotune``): tuning a hierarchy times every
candidate, keeps the heuristic among them, caches the choice per key, and changes no
result beyond the order of block reductions (solutions equal the untuned ones to 1e-12);
``stt_hier_tune`` rejects shapes outside its set."""

import numpy as np
import pytest
import torch

from conftest import rel_err
from oracle import sttopt_oracle as O

pytestmark = pytest.mark.gpu
EMIN, EMAX, PENAL = 1e-9, 1.0, 3.0


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_tuned_solve_equals_untuned(pkg, precision):
    from sttopt_b200 import _lib, autotune, torch_fem, torch_mg

    nelx, nely, rows = 192, 96, 4
    dev = torch.device("cuda")
    rng = np.random.default_rng(17)
    x = rng.uniform(1e-3, 1.0, (rows, nelx * nely))
    F, mask = O.cantilever_point_load(nelx, nely)
    args = (torch.tensor(O.simp_density(x, EMIN, EMAX, PENAL), device=dev),
            torch.tensor(O.element_dof_map(nelx, nely), device=dev), torch.tensor(O.plane_stress_KE(0.3), device=dev),
            torch.tensor(mask, device=dev), nelx, nely)
    b = torch_fem.project(torch.tensor(rng.standard_normal((rows, mask.size)), device=dev), args[3])
    try:
        autotune.disable()
        levels = torch_mg.build_hierarchy(*args, precision=precision)
        ref, n_ref = torch_fem.pcg(levels[0], b, torch_mg.VCycle(levels), rtol=1e-10)
        autotune.enable()
        levels = torch_mg.build_hierarchy(*args, precision=precision)
        got, n_got = torch_fem.pcg(levels[0], b, torch_mg.VCycle(levels), rtol=1e-10)
        entries = [v for k, v in autotune.cache().items() if f"{nelx}, {nely}" in k]
        assert entries and len(entries[-1]["ms"]) == len(autotune.PCG_BANDS) * len(autotune.LEVEL_WAVES)
        assert "0/0" in entries[-1]["ms"]  # the heuristic is a candidate
        assert rel_err(got.cpu(), ref.cpu()) < 1e-10 and abs(n_got - n_ref) <= 1
    finally:
        autotune.disable()
    h = levels[0]._hier
    for bad in [(12, 0), (8, -1), (8, 65)]:
        assert _lib.lib().stt_hier_tune(h.handle, *bad) == _lib.STT_ERR_INVALID
