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
