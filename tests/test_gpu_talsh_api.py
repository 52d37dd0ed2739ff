"""GPU: the talsh.h API end to end, replaying the reference's own driver tests
(TALSH/test.cpp test_talsh_c :38-147 and test_talsh_cxx :168-220) through
host-resident tensors, copy control, tasks and placement."""
import numpy as np
import pytest

import exatensor_b200.talsh as T
from exatensor_b200 import R8, C4

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def talsh():
    assert T.init((0,)) in (T.TALSH_SUCCESS, 1000001)
    yield T


def test_test_talsh_c_flow(talsh):
    d = T.Tensor([40, 40, 20, 20], R8, 0.0)
    l = T.Tensor([40, 40, 40, 40], R8, 0.001)
    r = T.Tensor([20, 40, 20, 40], R8, 0.01)
    task = T.Task()
    assert T.contract("D(a,b,i,j)+=L(c,b,d,a)*R(j,d,i,c)", d, l, r, 2.0, 0, T.DEV_NVIDIA_GPU, T.COPY_MTT, True,
                      task) == 0
    assert task.wait() == T.TALSH_TASK_COMPLETED
    total = task.time()[0]
    assert total > 0
    assert 1 in d.presence()            # COPY_M moved D to GPU 0 (flat id 1)
    d.place(0, T.DEV_HOST, T.COPY_M)    # back to the Host
    assert d.presence() == [0]
    assert abs(d.norm1_host() - 20480.0) <= 1e-9 * 20480.0
    assert l.presence() == [0] and r.presence() == [0]   # COPY_T kept inputs on the Host only


def test_test_talsh_cxx_flow(talsh):
    d = T.Tensor([40, 40, 20, 20], R8, 1.0)
    l = T.Tensor([20, 40, 20, 40], R8, 0.01)
    r = T.Tensor([40, 40, 40, 40], R8, 0.001)
    assert T.contract("D(a,b,c,d)+=L(d,i,c,j)*R(j,b,i,a)", d, l, r, 0.5, copy_ctrl=T.COPY_TTT,
                      accumulative=False) == 0
    assert np.allclose(d.host_array(), 0.01 * 0.001 * 40 * 40 * 0.5, rtol=1e-12)
    assert T.contract("D(a,b,c,d)+=L(d,i,c,j)*R(j,b,i,a)", d, l, r, 0.5, copy_ctrl=T.COPY_TTT) == 0
    assert np.allclose(d.host_array(), 0.01 * 0.001 * 40 * 40, rtol=1e-12)


def test_copy_add_with_external_memory(talsh):
    rng = np.random.default_rng(0)
    a = rng.uniform(-1, 1, 6 * 5 * 4)
    b = np.zeros(6 * 5 * 4)
    ta = T.Tensor([6, 5, 4], R8, ext=a)
    tb = T.Tensor([4, 6, 5], R8, ext=b)
    assert T.copy("D(c,a,b)=L(a,b,c)", tb, ta, copy_ctrl=T.COPY_TT) == 0
    ref = a.reshape(6, 5, 4, order="F").transpose(2, 0, 1).ravel(order="F")
    assert np.array_equal(b, ref)
    assert T.add("D(c,a,b)+=L(a,b,c)", tb, ta, 2.0, copy_ctrl=T.COPY_TT) == 0
    assert np.array_equal(b, ref + ref * 2.0)


def test_error_codes(talsh):
    d = T.Tensor([4, 4], R8)
    l = T.Tensor([4, 4], R8)
    r = T.Tensor([4, 4], R8)
    assert T.contract("D(a,b)+=L(k,a)*R(k,b)", d, l, r, dev_kind=T.DEV_HOST) == T.TALSH_NOT_AVAILABLE
    assert T.contract("D(a,b)+=L(k,a)*R(k,x)", d, l, r) == T.TALSH_INVALID_ARGS
    h = T.Tensor([4, 4, 4], R8)
    assert T.contract("D(a,b)+=L(a,k,b)*R(k,b)", d, h, r) == T.TALSH_NOT_IMPLEMENTED
    c = T.Tensor([4, 4], C4)
    assert T.contract("D(a,b)+=L(k,a)*R(k,b)", d, c, r) == T.TALSH_INVALID_ARGS


# ---- streamed contractions (host-resident inputs in slices) ----------------
def _fortran(x, dims):
    return x.reshape(dims, order="F")


def _contract_host(pattern, dd, ld, rd, l, r, d0, alpha, copy_ctrl, stream, dtk=R8):
    """Runs one contraction through talshTensorContract with host tensors
    (external memory) and returns D's host array; stream selects the sliced
    path (TB_STREAM_MIN_MB=0) or the ordinary one (TB_STREAM=0)."""
    import os
    env = {"TB_STREAM": None if stream else "0", "TB_STREAM_MIN_MB": "0" if stream else None}
    old = {k: os.environ.get(k) for k in env}
    for k, v in env.items():
        if v is None:
            os.environ.pop(k, None)
        else:
            os.environ[k] = v
    try:
        d = d0.copy()
        td, tl, tr = T.Tensor(dd, dtk, ext=d), T.Tensor(ld, dtk, ext=l), T.Tensor(rd, dtk, ext=r)
        assert T.contract(pattern, td, tl, tr, alpha, copy_ctrl=copy_ctrl) == 0
        return d, (td, tl, tr)
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_streamed_contraction_slices_left_operand(talsh):
    # V(a,b,c,d): its slowest index d is contracted, so V streams in contiguous
    # slices and T(c,d,i,j) in 2-D strided ones; D accumulates the slices
    rng = np.random.default_rng(5)
    v, o = 24, 8
    ld, rd, dd = [v, v, v, v], [v, v, o, o], [v, v, o, o]
    l = rng.uniform(-1, 1, int(np.prod(ld)))
    r = rng.uniform(-1, 1, int(np.prod(rd)))
    d0 = rng.uniform(-1, 1, int(np.prod(dd)))
    pat = "D(a,b,i,j)+=L(a,b,c,d)*R(c,d,i,j)"
    got, _ = _contract_host(pat, dd, ld, rd, l, r, d0, 0.75, T.COPY_TTT, stream=True)
    ref_dev, _ = _contract_host(pat, dd, ld, rd, l, r, d0, 0.75, T.COPY_TTT, stream=False)
    ref = d0 + 0.75 * np.einsum("abcd,cdij->abij", _fortran(l, ld), _fortran(r, rd)).ravel(order="F")
    assert _rel(got, ref) <= 1e-13
    assert _rel(got, ref_dev) <= 1e-13


def test_streamed_contraction_slices_right_operand(talsh):
    # L's slowest index is free, R's slowest (k) is contracted: R streams in
    # contiguous slices, L's slices are rows of a 2-D copy with inner extent 1
    rng = np.random.default_rng(6)
    ld, rd, dd = [50, 37], [41, 50], [37, 41]
    l = rng.uniform(-1, 1, 50 * 37)
    r = rng.uniform(-1, 1, 41 * 50)
    d0 = np.zeros(37 * 41)
    pat = "D(a,i)+=L(k,a)*R(i,k)"
    got, _ = _contract_host(pat, dd, ld, rd, l, r, d0, 1.0, T.COPY_TTT, stream=True)
    ref = np.einsum("ka,ik->ai", _fortran(l, ld), _fortran(r, rd)).ravel(order="F")
    assert _rel(got, ref) <= 1e-13


def test_streamed_contraction_complex_tensor_cores(talsh):
    # large enough for the tensor-core path per slice (M = N = K = 1296),
    # complex with a conjugated left operand; slices of d = 12 each
    from exatensor_b200 import C8
    rng = np.random.default_rng(7)
    n = 36
    ld, rd, dd = [n] * 4, [n] * 4, [n] * 4
    vol = n ** 4
    l = (rng.uniform(-1, 1, vol) + 1j * rng.uniform(-1, 1, vol)).astype(np.complex128)
    r = (rng.uniform(-1, 1, vol) + 1j * rng.uniform(-1, 1, vol)).astype(np.complex128)
    d0 = np.zeros(vol, dtype=np.complex128)
    pat = "D(a,b,i,j)+=L+(a,b,c,d)*R(c,d,i,j)"
    got, _ = _contract_host(pat, dd, ld, rd, l, r, d0, 1.0, T.COPY_TTT, stream=True, dtk=C8)
    ref_dev, _ = _contract_host(pat, dd, ld, rd, l, r, d0, 1.0, T.COPY_TTT, stream=False, dtk=C8)
    ref = np.einsum("abcd,cdij->abij", np.conj(_fortran(l, ld)), _fortran(r, rd)).ravel(order="F")
    assert _rel(got, ref) <= 1e-12
    assert _rel(ref_dev, ref) <= 1e-12


def test_streamed_contraction_discards_inputs_on_copy_d(talsh):
    rng = np.random.default_rng(8)
    ld, rd, dd = [16, 16, 12], [12, 10], [16, 16, 10]
    l = rng.uniform(-1, 1, 16 * 16 * 12)
    r = rng.uniform(-1, 1, 120)
    d0 = np.zeros(16 * 16 * 10)
    copy_tdt = (T.COPY_T << 4) | (T.COPY_D << 2) | T.COPY_T
    got, (td, tl, tr) = _contract_host("D(a,b,i)+=L(a,b,k)*R(k,i)", dd, ld, rd, l, r, d0, 1.0, copy_tdt,
                                       stream=True)
    ref = np.einsum("abk,ki->abi", _fortran(l, ld), _fortran(r, rd)).ravel(order="F")
    assert _rel(got, ref) <= 1e-13
    assert tl.presence() == [] and tr.presence() == [0]


def test_streamed_contraction_uneven_slices(talsh):
    # extent 7 in three slices of 3, 3 and 1
    rng = np.random.default_rng(9)
    ld, rd, dd = [30, 20, 7], [7, 25], [30, 20, 25]
    l = rng.uniform(-1, 1, 30 * 20 * 7)
    r = rng.uniform(-1, 1, 7 * 25)
    d0 = rng.uniform(-1, 1, 30 * 20 * 25)
    got, _ = _contract_host("D(a,b,i)+=L(a,b,k)*R(k,i)", dd, ld, rd, l, r, d0, -1.5, T.COPY_TTT, stream=True)
    ref = d0 - 1.5 * np.einsum("abk,ki->abi", _fortran(l, ld), _fortran(r, rd)).ravel(order="F")
    assert _rel(got, ref) <= 1e-13


# ---- output decomposition (talshTensorContractXL with D beyond the budget) --
def _contract_xl(pattern, dd, ld, rd, l, r, d0, alpha, accumulative, budget_mb, dtk=R8):
    """talshTensorContractXL with host tensors under a device budget of
    budget_mb (TB_XL_DEVICE_MB); returns D and the split it reported."""
    import os
    old = os.environ.get("TB_XL_DEVICE_MB")
    os.environ["TB_XL_DEVICE_MB"] = str(budget_mb)
    try:
        d = d0.copy()
        td, tl, tr = T.Tensor(dd, dtk, ext=d), T.Tensor(ld, dtk, ext=l), T.Tensor(rd, dtk, ext=r)
        assert T.contract_xl(pattern, td, tl, tr, alpha, accumulative=accumulative) == 0
        return d, T.xl_last_split()
    finally:
        if old is None:
            os.environ.pop("TB_XL_DEVICE_MB", None)
        else:
            os.environ["TB_XL_DEVICE_MB"] = old


@pytest.mark.parametrize("accumulative", [True, False])
def test_xl_decomposes_the_output_beyond_the_budget(talsh, accumulative):
    # D and L are 42 MB each, R 2.6 MB: under a 64 MB budget D is cut along
    # b (extent 96, the slowest of the largest), which L carries
    rng = np.random.default_rng(11)
    v, o = 96, 24
    ld, rd, dd = [v, v, o, o], [o, o, o, o], [v, v, o, o]
    l = rng.uniform(-1, 1, int(np.prod(ld)))
    r = rng.uniform(-1, 1, int(np.prod(rd)))
    d0 = rng.uniform(-1, 1, int(np.prod(dd)))
    pat = "D(a,b,i,j)+=L(a,b,c,d)*R(c,d,i,j)"
    got, split = _contract_xl(pat, dd, ld, rd, l, r, d0, 0.5, accumulative, 64)
    assert split[0] == 1 and split[1] >= 4, split
    prod = 0.5 * np.einsum("abcd,cdij->abij", _fortran(l, ld), _fortran(r, rd)).ravel(order="F")
    ref = d0 + prod if accumulative else prod
    assert _rel(got, ref) <= 1e-12
    if accumulative:  # the undecomposed contraction of the same tensors
        whole, _ = _contract_host(pat, dd, ld, rd, l, r, d0, 0.5, T.COPY_TTT, stream=False)
        assert _rel(got, whole) <= 1e-12


def test_xl_decomposes_along_the_right_operand_complex(talsh):
    # the largest D extent (j = 80) comes from R; complex data, conjugated L
    from exatensor_b200 import C8
    rng = np.random.default_rng(12)
    ld, rd, dd = [20, 30, 16], [16, 40, 80], [20, 30, 40, 80]
    cplx = lambda n: rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
    l, r = cplx(int(np.prod(ld))), cplx(int(np.prod(rd)))
    d0 = cplx(int(np.prod(dd)))
    pat = "D(a,b,i,j)+=L+(a,b,k)*R(k,i,j)"
    got, split = _contract_xl(pat, dd, ld, rd, l, r, d0, 1.0, True, 24, dtk=C8)
    assert split[0] == 3 and split[1] >= 2, split
    ref = d0 + np.einsum("abk,kij->abij", np.conj(_fortran(l, ld)), _fortran(r, rd)).ravel(order="F")
    assert _rel(got, ref) <= 1e-12
