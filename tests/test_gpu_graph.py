"""The single-image CUDA-graph entry (pipeline_<name>_graph): captured on
the first call, replayed after, re-captured when the parameters change; it
must read the inputs' current contents on every replay.  Tolerances as in
the single-call parity tests (Harris 1e-5 relative, bilateral 1e-5,
pyramid 2e-5).  The camera pipe computes its const tables from input
contents on the host, so it has no graph form."""

import numpy as np
import pytest

import oracle.bilateral as OB
import oracle.campipe as OC
import oracle.harris as OH
import oracle.pyramid as OP
from polymage_b200.apps import catalog
from polymage_b200.runtime import PipelineRuntimeError
from tests import pipelines

pytestmark = pytest.mark.gpu


def test_harris_graph_replays_and_recaptures(cuda):
    import torch
    cp = pipelines.harris()
    for rows, cols, seeds in [(300, 420, (1, 2)), (515, 771, (3,)),
                              (300, 420, (4,))]:
        t_in = torch.empty((rows, cols), dtype=torch.float32, device=cuda)
        out = torch.zeros((rows, cols), dtype=torch.float32, device=cuda)
        for seed in seeds:
            img = OH.make_input(rows, cols, seed=seed)
            t_in.copy_(torch.from_numpy(img))
            out.zero_()
            cp.run_dev({'R': rows - 2, 'C': cols - 2}, {'img': t_in},
                       {'harris': out}, graph=True)
            torch.cuda.synchronize()
            cp.check()
            ref = OH.harris(img)
            err = np.abs(out.cpu().numpy() - ref).max() / np.abs(ref).max()
            assert err <= 1e-5, err


def test_bilateral_and_pyramid_graph(cuda):
    import torch
    cb = catalog.build("bilateral")
    img = OB.make_input(700, 333, seed=9)
    out = torch.zeros((1, 700, 333), dtype=torch.float32, device=cuda)
    for _ in range(2):                 # the grid is re-initialized
        cb.run_dev({'rows': 700, 'cols': 333},
                   {'input': torch.from_numpy(img).to(cuda)},
                   {'filtered': out}, graph=True)
        torch.cuda.synchronize()
        cb.check()
        assert np.abs(out.cpu().numpy() - OB.bilateral(img)).max() <= 1e-5
    cpy = catalog.build("pyramid")
    R, C = 157, 211
    img1, img2, mask = OP.make_inputs(R, C, seed=5)
    (x0, x1), (y0, y1) = OP.output_box(R, C)
    o = torch.zeros((3, x1 - x0 + 1, y1 - y0 + 1), dtype=torch.float32,
                    device=cuda)
    cpy.run_dev({'R': R, 'C': C}, {'img1': torch.from_numpy(img1).to(cuda),
                                   'img2': torch.from_numpy(img2).to(cuda),
                                   'mask': torch.from_numpy(mask).to(cuda)},
                {'blend': o}, graph=True)
    torch.cuda.synchronize()
    cpy.check()
    ref = OP.pyramid_blend(img1, img2, mask)
    assert np.abs(o.cpu().numpy().astype(np.float64) - ref).max() <= 2e-5


def test_campipe_has_no_graph_form(cuda):
    import torch
    cp = catalog.build("campipe")
    R, C = 256, 384
    img = OC.make_input(R, C, seed=3)
    out = torch.zeros((3, R - 48, C - 64), dtype=torch.uint8, device=cuda)
    prm = {'C': C, 'R': R, 'colour_temp': 3700.0, 'contrast': 50.0,
           'gamma': 2.0}
    ins = {'img': torch.from_numpy(img).to(cuda),
           'matrix_3200': torch.from_numpy(OC.MATRIX_3200).to(cuda),
           'matrix_7000': torch.from_numpy(OC.MATRIX_7000).to(cuda)}
    with pytest.raises(PipelineRuntimeError):
        cp.run_dev(prm, ins, {'process': out}, graph=True)
    cp.run_dev(prm, ins, {'process': out})          # the stream entry works
    torch.cuda.synchronize()
    cp.check()
    assert np.array_equal(out.cpu().numpy(), OC.campipe(img, 3700.0, 50.0,
                                                        2.0))
