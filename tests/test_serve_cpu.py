"""Host-side logic of the serving loop (no GPU): request streams, footprints, classes."""
import numpy as np

from fosite_b200 import abi
from fosite_b200.serve import Request, build_problem, footprint_bytes, kernel_class, poisson_stream


def test_poisson_stream_shapes_and_rates():
    reqs = poisson_stream(rate=200.0, n=400, seed=3)
    t = np.array([r.arrival for r in reqs])
    assert np.all(np.diff(t) > 0)
    assert abs(len(reqs) / t[-1] - 200.0) < 40.0
    for r in reqs:
        if r.kind == "khi":
            assert 64 <= r.size[0] <= 1024 and r.size[0] == r.size[1]
        elif r.kind == "disk":
            assert 64 <= r.size[0] <= 512 and r.size[1] == 2 * r.size[0]
        else:
            assert 32 <= r.size[0] <= 128 and len(r.size) == 3
        assert r.t_end > 0
    assert {r.kind for r in reqs} == {"khi", "disk", "pulse"}


def test_footprint_grows_with_the_grid():
    a = footprint_bytes(build_problem(Request("khi", (64, 64), 0.1))[0])
    b = footprint_bytes(build_problem(Request("khi", (128, 128), 0.1))[0])
    assert 3.5 * a < b < 4.5 * a
    c = footprint_bytes(build_problem(Request("pulse", (32, 32, 32), 0.1))[0])
    assert c > 3 * 5 * 8 * 32 ** 3


def test_kernel_classes_group_compatible_requests():
    k1 = kernel_class(build_problem(Request("disk", (64, 128), 0.1, seed=1))[0])
    k2 = kernel_class(build_problem(Request("disk", (128, 256), 0.1, seed=2))[0])
    k3 = kernel_class(build_problem(Request("khi", (64, 64), 0.1))[0])
    k4 = kernel_class(build_problem(Request("pulse", (32, 32, 32), 0.1))[0])
    assert k1 == k2 and len({k1, k3, k4}) == 3
    cfg = build_problem(Request("pulse", (32, 32, 32), 0.25))[0]
    assert cfg.method == abi.DORMAND_PRINCE and cfg.stoptime == 0.25   # configs: the pulse is DOPRI
