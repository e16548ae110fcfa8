"""GPU parity of the pipelines beyond the five benchmark configurations:
pyramid interpolation, Jacobi 2-D and 3-D, the multigrid V- and W-cycles
in 2-D and 3-D, and the NAS MG V-cycle, each against its FP64 restatement
(oracle/interpolate.py, jacobi.py, multigrid.py, nas_mg.py), through the
reference's host-buffer C ABI and through the device entry.

Builds: the catalog's, at the reference Makefiles' settings (Jacobi 10
steps; cycles with 3 levels, 10 pre-smoothings and none after or on the
coarsest grid; NAS MG class W), plus the reference arg parsers' defaults
for the cycles (2 levels, one smoothing at each place) and NAS MG class S.
A built library accepts any size at run time; the sizes below include odd
ones.

Tolerances: float64 pipelines max |gpu - ref| <= 1e-10 * max(1, max|ref|)
(FMA contraction and summation order only); float32 interpolation
max |gpu - ref| <= 1e-5 (outputs are ratios in [0, ~1]).  Outputs are
zero-filled first: points the spec does not write stay 0, as in the
restatements."""

import numpy as np
import pytest

import oracle.interpolate as OI
import oracle.jacobi as OJ
import oracle.multigrid as OM
import oracle.nas_mg as ON
from polymage_b200.apps import catalog

pytestmark = pytest.mark.gpu


def _f64_close(out, ref):
    err = np.abs(out - ref).max()
    assert err <= 1e-10 * max(1.0, np.abs(ref).max()), err


def _host(cp, params, inputs, out_shapes):
    outs = dict((k, np.zeros(s, dt)) for k, (s, dt) in out_shapes.items())
    cp.run_host(params, inputs, outs)
    return outs


@pytest.mark.parametrize("R,C", [(128, 160), (211, 157), (2048, 2048)])
def test_interpolate(R, C):
    cp = catalog.build("interpolate")
    img = OI.make_input(R, C, seed=R + C)
    out = _host(cp, {'R': R, 'C': C}, {'img': img},
                {'interpolate': ((3, R, C), np.float32)})['interpolate']
    ref = OI.interpolate(img)
    assert np.abs(out.astype(np.float64) - ref).max() <= 1e-5


@pytest.mark.parametrize("N", [200, 333, 2048])
def test_jacobi2d(N):
    cp = catalog.build("jacobi2d")
    V, F = OJ.make_input(N, seed=N)
    out = _host(cp, {'N': N}, {'V_': V, 'F_': F},
                {'jacobi': ((N + 2, N + 2), np.float64)})['jacobi']
    _f64_close(out, OJ.jacobi2d(V, F, T=catalog.JACOBI2D['T']))


@pytest.mark.parametrize("N", [30, 47, 128])
def test_jacobi3d(N):
    cp = catalog.build("jacobi3d")
    V = np.random.default_rng(N).random((N + 2,) * 3)
    F = np.random.default_rng(N + 1).random((N + 2,) * 3)
    out = _host(cp, {'N': N}, {'V_': V, 'F_': F},
                {'jacobi': ((N + 2,) * 3, np.float64)})['jacobi']
    _f64_close(out, OJ.jacobi3d(V, F, T=catalog.JACOBI3D['T']))


_CYCLES = {
    # catalog name: (oracle, input maker, dims)
    "vcycle": (OM.v_cycle, OM.make_input, 2),
    "wcycle": (OM.v_cycle, OM.make_input, 2),
    "vcycle3d": (OM.v_cycle3d, OM.make_input3d, 3),
    "wcycle3d": (OM.v_cycle3d, OM.make_input3d, 3),
}


def _cycle_case(cp, name, kw, n, seed):
    oracle, make, dims = _CYCLES[name]
    L = kw['L']
    V, F = make(n, L=L, seed=seed)
    N = V.shape[0] - 2
    out = _host(cp, {'n': n}, {'V_': V, 'F_': F},
                {cp.outputs[0].name: ((N + 2,) * dims, np.float64)})
    ref = oracle(V, F, n, L=L, nu1=kw['nu1'], nu2=kw['nu2'], nuc=kw['nuc'],
                 gamma=kw.get('gamma', 1))
    _f64_close(out[cp.outputs[0].name], ref)


@pytest.mark.parametrize("name,n", [("vcycle", 31), ("vcycle", 20),
                                    ("wcycle", 31), ("wcycle", 13),
                                    ("vcycle3d", 15), ("vcycle3d", 8),
                                    ("wcycle3d", 15), ("wcycle3d", 6)])
def test_multigrid_cycles(name, n):
    """The reference Makefiles' cycles (L=3, nu1=10, nu2=nuc=0)."""
    kw = dict(catalog._BUILDERS[name][1])
    _cycle_case(catalog.build(name), name, kw, n, seed=n)


@pytest.mark.parametrize("gamma,dims", [(1, 2), (2, 2), (1, 3)])
def test_multigrid_cycles_with_post_and_coarse_smoothing(gamma, dims):
    """The reference arg parsers' defaults: L=2, one pre-, post- and
    coarse-grid smoothing."""
    from polymage_b200.apps.multigrid import build_v_cycle
    name = {(1, 2): "vcycle", (2, 2): "wcycle", (1, 3): "vcycle3d"}[
        (gamma, dims)]
    kw = dict(n=15 if dims == 2 else 7, L=2, nu1=1, nu2=1, nuc=1,
              gamma=gamma, dims=dims,
              tile_sizes=(16, 64) if dims == 2 else (4, 8, 32),
              name={"vcycle": "Vcycle_d", "wcycle": "Wcycle_d",
                    "vcycle3d": "Vcycle3d_d"}[name])
    cp = build_v_cycle(**kw).build()
    for n in ((15, 22) if dims == 2 else (7, 10)):
        _cycle_case(cp, name, kw, n, seed=n)


@pytest.mark.parametrize("prob_class,n", [("S", 32), ("W", 128)])
def test_nas_mg(prob_class, n):
    from polymage_b200.apps.nas_mg import build_mg3p
    cp = catalog.build("mg3p") if prob_class == "W" else \
        build_mg3p('S').build()
    U, V, R = ON.make_input(n, seed=n)
    outs = _host(cp, {'n': n}, {'U': U, 'V': V, 'R': R},
                 {'MG_U': ((n + 2,) * 3, np.float64),
                  'MG_R': ((n + 2,) * 3, np.float64)})
    ru, rr = ON.mg3p(U, V, R, prob_class=prob_class)
    _f64_close(outs['MG_U'], ru)
    _f64_close(outs['MG_R'], rr)


def test_device_entry_matches_host_entry(cuda):
    """The device-buffer entry (``_dev``, caller's stream) gives the host
    entry's result for a float64 pipeline and the float32 one."""
    import torch
    cp = catalog.build("jacobi2d")
    N = 257
    V, F = OJ.make_input(N, seed=3)
    out = torch.zeros((N + 2, N + 2), dtype=torch.float64, device=cuda)
    cp.run_dev({'N': N}, {'V_': torch.from_numpy(V).to(cuda),
                          'F_': torch.from_numpy(F).to(cuda)},
               {'jacobi': out})
    torch.cuda.synchronize()
    cp.check()
    _f64_close(out.cpu().numpy(), OJ.jacobi2d(V, F, T=catalog.JACOBI2D['T']))
    cp = catalog.build("interpolate")
    img = OI.make_input(300, 200, seed=4)
    out = torch.zeros((3, 300, 200), dtype=torch.float32, device=cuda)
    cp.run_dev({'R': 300, 'C': 200}, {'img': torch.from_numpy(img).to(cuda)},
               {'interpolate': out})
    torch.cuda.synchronize()
    cp.check()
    assert np.abs(out.cpu().numpy() - OI.interpolate(img)).max() <= 1e-5
