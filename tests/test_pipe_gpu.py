"""GPU tests of the FP16S async-copy pipeline (flb_set_launch ctas_per_sm = -1,
k_pull_pipe): its updates are bit-for-bit those of the direct kernel, on the
cavity and on lattices whose row ends, padding and interior-row limits fall
everywhere within a warp's tile."""
import numpy as np
import pytest

import freelb_b200 as F
from conftest import rel_maxnorm
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def random_lattice(nx, ny, nz, model, seed, tau=0.56):
    """Flags drawn from {void, fluid, wall, lid} so that every op pairs with every
    other in a cell pair; lid cells get a seeded wall velocity."""
    rng = np.random.default_rng(seed)
    lat = F.Lattice(nx, ny, nz, tau, storage="fp16s", model=model)
    flags = rng.choice(np.array([1, 2, 4, 8], dtype=np.uint8), size=lat.N, p=[0.1, 0.6, 0.2, 0.1])
    lat.upload_flags(flags)
    u = np.zeros((lat.N, 3), dtype=lat.real)
    u[flags == 8] = rng.uniform(-0.05, 0.05, size=(int((flags == 8).sum()), 3))
    lat.upload_field("u", u)
    return lat


def run_both(make, steps):
    out = []
    for ctas in (0, -1):
        lat = make()
        lat.set_launch(4, ctas, 4)
        lat.step(steps)
        out.append(lat.download_pops())
        lat.close()
    return out


@pytest.mark.parametrize("model", ["bgk", "mrt", "les"])
@pytest.mark.parametrize("ni", [10, 21, 30, 62])
def test_pipe_equals_direct_kernel_on_cavity(gpu_ok, model, ni):
    a, b = run_both(lambda: F.cavity(ni, tau=0.55, storage="fp16s", model=model), 25)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("model", ["bgk", "mrt", "les"])
@pytest.mark.parametrize("dims", [(3, 5, 7), (5, 7, 6), (14, 9, 7), (33, 6, 9), (66, 5, 5),
                                  (130, 4, 6), (250, 4, 5)])
def test_pipe_equals_direct_kernel_on_random_flags(gpu_ok, model, dims):
    a, b = run_both(lambda: random_lattice(*dims, model, seed=sum(dims)), 12)
    assert np.array_equal(a, b)


def test_pipe_matches_oracle(gpu_ok):
    lat = F.cavity(21, tau=0.55, storage="fp16s")
    lat.set_launch(4, -1, 4)
    lat.step(30)
    ref = O.cavity(21, tau=0.55, dtype=np.float64)
    ref.step(30)
    assert rel_maxnorm(lat.download_pops(), ref.pops) < 2e-3


def test_pipe_graph_equals_plain(gpu_ok):
    a = F.cavity(30, storage="fp16s")
    b = F.cavity(30, storage="fp16s")
    a.set_launch(4, -1, 4)
    b.set_launch(4, -1, 4)
    a.step(7, graph=True)
    b.step(7)
    assert np.array_equal(a.download_pops(), b.download_pops())


def test_pipe_launch_rules(gpu_ok):
    with pytest.raises(F.FlbError):
        F.cavity(8, storage="fp32").set_launch(4, -1, 4)
    with pytest.raises(F.FlbError):
        F.cavity(8, storage="fp64").set_launch(4, -1, 2)
    with pytest.raises(F.FlbError):
        F.cavity(8, storage="fp16s").set_launch(4, -1, 2)  # 4 cells per thread only
    lat = F.cavity(8, storage="fp16s")
    lat.set_launch(4, -1, 0)
    assert lat.get_launch() == (4, -1, 4)
