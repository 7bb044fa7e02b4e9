"""The halo pack / unpack launch (redi_b200_halo_copy) against torch slicing, on one GPU.

The multi-rank exchange itself is tested on CPU ranks (test_halo_gloo.py); here the
library launch that packs a tile column or row of every field into a neighbour's buffer,
and unpacks a received buffer into the ghost column or row, must move exactly the values
that slicing the (nz, ny, nx) arrays names, in the same order.
"""

import ctypes as C

import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU-only container
    pytest.skip("needs a CUDA device", allow_module_level=True)


def _copy(R, fields, axis, index, buf, to_buf):
    L = R.lib()
    L.redi_b200_halo_copy.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                      C.c_void_p, C.c_int, C.c_void_p]
    nz, ny, nx = fields[0].shape
    ptrs = (C.c_void_p * len(fields))(*[t.data_ptr() for t in fields])
    return L.redi_b200_halo_copy(ptrs, len(fields), nx, ny, nz, axis, index, buf.data_ptr(), int(to_buf), None)


@pytest.mark.parametrize("axis,index", [(0, 2), (0, 38), (1, 2), (1, 24)])
def test_pack_and_unpack_match_slicing(redi_lib, axis, index):
    R = redi_lib
    g = torch.Generator(device="cuda").manual_seed(3)
    nz, ny, nx = 7, 27, 41
    fields = [torch.randn(nz, ny, nx, dtype=torch.float64, device="cuda", generator=g) for _ in range(3)]
    sl = (slice(None), slice(None), index) if axis == 0 else (slice(None), index, slice(None))
    n = nz * (ny if axis == 0 else nx)
    buf = torch.empty(3 * n, dtype=torch.float64, device="cuda")
    assert _copy(R, fields, axis, index, buf, True) == R.OK
    torch.cuda.synchronize()
    ref = torch.cat([t[sl].reshape(-1) for t in fields])
    assert torch.equal(buf, ref)
    incoming = torch.randn(3 * n, dtype=torch.float64, device="cuda", generator=g)
    before = [t.clone() for t in fields]
    assert _copy(R, fields, axis, index, incoming, False) == R.OK
    torch.cuda.synchronize()
    for f, (t, b) in enumerate(zip(fields, before)):
        exp = b.clone()
        exp[sl] = incoming[f * n:(f + 1) * n].view(exp[sl].shape)
        assert torch.equal(t, exp), f


def test_bad_arguments_are_refused(redi_lib):
    R = redi_lib
    t = torch.zeros(2, 3, 4, dtype=torch.float64, device="cuda")
    buf = torch.zeros(100, dtype=torch.float64, device="cuda")
    assert _copy(R, [t], 0, 4, buf, True) == R.E_ARG  # index beyond nx
    assert _copy(R, [t], 2, 0, buf, True) == R.E_ARG  # no such axis
