"""akb_kinetic_energy_static: the kinetic energy of a model's device arrays
computed without allocating device memory (for callers that cannot call
cudaMalloc mid-run: inside CUDA stream capture, or under a device-memory
budget owned by another allocator). Checked against akb_get_energy on two
consecutive calls, against a float64 torch sum on inputs of one to the maximum
2048 partial blocks, inside a captured CUDA graph on a side stream, and for
device memory left unchanged by a call. Collected last so that a failure here
leaves every other test already run."""
import ctypes as C

import numpy as np
import pytest

from akantu_b200 import _abi, configs
from tests.golden_cases import GpuAdapter

pytestmark = pytest.mark.gpu

MAX_NODES = 8388608  # 2048 partial blocks of 256 threads x 16 nodes


def _call(mass, vel, nn, dim, out, stream=None):
    from akantu_b200._lib import lib
    return lib().akb_kinetic_energy_static(C.c_void_p(mass), C.c_void_p(vel), nn, dim,
                                           C.c_void_p(out), stream)


def static_kinetic(model, out_tensor):
    from akantu_b200._lib import check
    dim = model.m.dim
    nn = model.m.mesh.getNbNodes()
    mass = model.m.devicePointer(_abi.FIELD_MASS)
    vel = model.m.devicePointer(_abi.FIELD_VELOCITY)
    model.m.synchronize()
    check(_call(mass, vel, nn, dim, out_tensor.data_ptr()))
    import torch
    torch.cuda.synchronize()
    return float(out_tensor.item())


def test_static_kinetic_energy_matches_model_on_two_calls():
    import torch
    w = configs.cube_tet4(n=10)
    model = GpuAdapter(w["mesh"], w["materials"], precision=_abi.MODE_FP64)
    configs.setup_model(model, w)
    out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    results = []
    for steps in (7, 13):
        model.solve_steps(steps)
        ref = model.energy(_abi.ENERGY_KINETIC)
        got = static_kinetic(model, out)
        assert ref > 0
        assert abs(got - ref) <= 1e-12 * ref, (got, ref)
        results.append(got)
    assert results[0] != results[1]  # the second call saw the new state


def _synthetic(nn, dim, seed):
    """Masses in (0, 2] with about 10 % of the components at zero or at
    DBL_EPSILON (both excluded from the sum, like massless components in
    getKineticEnergy), velocities N(0, 1)."""
    import torch
    g = torch.Generator(device="cuda").manual_seed(seed)
    m = torch.rand(nn, dim, dtype=torch.float64, device="cuda", generator=g) * 2
    drop = torch.rand(nn, dim, device="cuda", generator=g) < 0.1
    m[drop] = 0.0
    m[drop & (torch.rand(nn, dim, device="cuda", generator=g) < 0.5)] = np.finfo(np.float64).eps
    v = torch.randn(nn, dim, dtype=torch.float64, device="cuda", generator=g)
    ref = 0.5 * float((v * v * torch.where(m > np.finfo(np.float64).eps, m, 0)).sum())
    return m, v, ref


@pytest.mark.parametrize("nn,dim", [(1, 3), (4097, 2), (100003, 3), (MAX_NODES - 5, 1),
                                    (MAX_NODES, 1)])
def test_static_kinetic_energy_on_several_blocks(nn, dim):
    """One block, a block and a node, ~25 blocks, and the full 2048 blocks,
    where the finishing pass reduces 8 partials per thread."""
    import torch
    from akantu_b200._lib import check
    m, v, ref = _synthetic(nn, dim, seed=nn)
    out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    check(_call(m.data_ptr(), v.data_ptr(), nn, dim, out.data_ptr()))
    torch.cuda.synchronize()
    assert abs(out.item() - ref) <= 1e-12 * ref, (out.item(), ref)


def test_static_kinetic_energy_in_a_captured_graph_allocates_nothing():
    """A warm-up call, then the call captured into a CUDA graph on a side
    stream and replayed after the velocities change: each replay sees the
    current arrays, and neither the call nor the replays change the free
    device memory."""
    import torch
    from akantu_b200._lib import check
    nn, dim = 300007, 3
    m, v, ref = _synthetic(nn, dim, seed=11)
    out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    side = torch.cuda.Stream()
    check(_call(m.data_ptr(), v.data_ptr(), nn, dim, out.data_ptr(), C.c_void_p(side.cuda_stream)))
    torch.cuda.synchronize()
    assert abs(out.item() - ref) <= 1e-12 * ref
    free0 = torch.cuda.mem_get_info()[0]
    check(_call(m.data_ptr(), v.data_ptr(), nn, dim, out.data_ptr(), C.c_void_p(side.cuda_stream)))
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.stream(side):
        graph.capture_begin()
        check(_call(m.data_ptr(), v.data_ptr(), nn, dim, out.data_ptr(),
                    C.c_void_p(side.cuda_stream)))
        graph.capture_end()
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    for scale in (2.0, 0.5):
        v.mul_(scale)
        ref *= scale * scale
        out.fill_(-1.0)
        torch.cuda.synchronize()
        graph.replay()
        torch.cuda.synchronize()
        assert abs(out.item() - ref) <= 1e-12 * ref, (out.item(), ref)
        assert torch.cuda.mem_get_info()[0] == free1
    del graph


def test_static_kinetic_energy_rejects_oversize():
    from akantu_b200._lib import lib
    L = lib()
    dummy = C.c_void_p(1)  # never dereferenced: the size check comes first
    st = L.akb_kinetic_energy_static(dummy, dummy, MAX_NODES + 1, 3, dummy, None)
    assert st == _abi.AKB_ERR_INVALID_ARGUMENT
    assert b"8388608" in L.akb_last_error()
