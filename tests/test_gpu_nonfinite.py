"""GPU parity: NaN and infinities in the operands propagate through every
contraction method the way the reference's cuBLAS GEMM propagates them
(TALSH/tensor_algebra_gpu_nvidia.cu:6899-7024, an IEEE GEMM): an entry of D
whose dot product meets a NaN, an infinity times zero, or infinities of both
signs is NaN; one that meets infinities of one sign is that infinity.

On the tensor-core path the operand preparation flags rows and columns that
hold a non-finite value, the GEMM epilogue leaves their D entries alone, and a
fix-up kernel computes them as plain FP64 dot products.  The test plants NaN,
+Inf, -Inf, and Inf-times-zero cases in L rows and R columns of a contraction
large enough for METHOD_AUTO to take the tensor-core path, and checks:
  * the NaN / +Inf / -Inf pattern of D equals the IEEE pattern exactly;
  * the finite entries are within the method's tolerance of an FP64 reference
    (relative Frobenius: 1e-12 for R8/C8, 1e-4 for R4/C4 on the tensor cores;
    1e-13 / 2e-5 for plain TTGT).
"""
import numpy as np
import pytest

import exatensor_b200 as XB
import oracle as O
from tests.test_gpu_permute import rand_host

pytestmark = pytest.mark.gpu
PATTERN = "D(i,j)+=L(k,i)*R(k,j)"
M, N, K = 1536, 1280, 2048   # 2*M*N*K = 8.1e9 FLOP: METHOD_AUTO takes the tensor cores
TOL = {(XB.METHOD_FUSED, O.R8): 1e-12, (XB.METHOD_FUSED, O.C8): 1e-12, (XB.METHOD_FUSED, O.R4): 1e-4,
       (XB.METHOD_FUSED, O.C4): 1e-4, (XB.METHOD_TTGT, O.R8): 1e-13, (XB.METHOD_TTGT, O.C8): 1e-13,
       (XB.METHOD_TTGT, O.R4): 2e-5, (XB.METHOD_TTGT, O.C4): 2e-5}


def plant(dtk):
    """L as (M, K) and R as (N, K) row-major views of the dlf tensors L(k,i),
    R(k,j), with non-finite values planted in a few rows of L and columns of R."""
    cplx = dtk in (O.C4, O.C8)
    L = rand_host(dtk, M * K, 31).reshape(M, K)
    R = rand_host(dtk, N * K, 32).reshape(N, K)
    inf, nan = np.inf, np.nan
    L[5, 7] = nan                       # row 5: NaN everywhere
    L[100, 3] = inf                     # row 100: +-Inf by the sign of R(3, j) ...
    R[50, 3] = 0.0                      # ... and Inf * 0 = NaN in column 50
    L[200, 1], L[200, 2] = inf, -inf    # row 200: NaN where R(1, j), R(2, j) share a sign
    R[9, 4] = -inf                      # column 9
    R[17, 0] = nan                      # column 17
    L[M - 1, K - 1] = -inf              # the last row, last k (edge of the padded tiles)
    if cplx:
        L[300, 11] = complex(0.25, inf)  # an infinite imaginary part
        R[33, 12] = complex(nan, 0.5)    # a NaN real part
    return L, R


def ieee_reference(L, R, D0, alpha, accumulative):
    """D as (N, M): clean entries by an FP64 matrix product, entries of flagged
    rows / columns by direct IEEE dot products (order does not change which
    non-finite value results)."""
    cplx = np.iscomplexobj(L)
    Lw = L.astype(np.complex128 if cplx else np.float64)
    Rw = R.astype(np.complex128 if cplx else np.float64)
    bad_r = ~np.isfinite(Lw).all(axis=1)
    bad_c = ~np.isfinite(Rw).all(axis=1)
    Lc = np.where(bad_r[:, None], 0, Lw)
    Rc = np.where(bad_c[:, None], 0, Rw)
    out = Rc @ Lc.T                                     # (N, M)
    with np.errstate(invalid="ignore", over="ignore"):
        def dots(x, Y):  # IEEE dot products x . Y[j], real and imaginary parts separately
            if not cplx:
                return (Y * x).sum(axis=1)
            re = (Y.real * x.real).sum(axis=1) - (Y.imag * x.imag).sum(axis=1)
            im = (Y.real * x.imag).sum(axis=1) + (Y.imag * x.real).sum(axis=1)
            return re + 1j * im
        for i in np.nonzero(bad_r)[0]:
            out[:, i] = dots(Lw[i], Rw)
        for j in np.nonzero(bad_c)[0]:
            out[j, :] = dots(Rw[j], Lw)
        ref = alpha * out
        if accumulative:
            ref = ref + D0.reshape(N, M)
    return ref


def classes(x):
    parts = [x.real, x.imag] if np.iscomplexobj(x) else [x]
    return [(np.isnan(p), np.isposinf(p), np.isneginf(p)) for p in parts]


def run(xt, dev, dtk, method, accumulative, alpha):
    L, R = plant(dtk)
    D0 = rand_host(dtk, M * N, 33)
    dd, ld, rd = dev.put(D0), dev.put(L.ravel()), dev.put(R.ravel())
    xt.tensor_contract(PATTERN, dtk, [M, N], dd.data_ptr(), [K, M], ld.data_ptr(), [K, N], rd.data_ptr(), alpha,
                       accumulative=accumulative, plan=xt.make_plan(method), stream=dev.stream())
    got = dev.get(dd, D0.dtype, D0.size).reshape(N, M)
    xt.device_check(dev.stream())
    st = xt.last_contract_stats()
    ref = ieee_reference(L, R, D0, alpha, accumulative)
    return got, ref, st


@pytest.mark.parametrize("dtk", [O.R8, O.R4, O.C8, O.C4])
@pytest.mark.parametrize("method", [XB.METHOD_AUTO, XB.METHOD_FUSED, XB.METHOD_TTGT])
def test_nonfinite_propagation(xt, dev, dtk, method):
    for accumulative, alpha in ((True, 0.5), (False, -1.5)):
        got, ref, st = run(xt, dev, dtk, method, accumulative, alpha)
        if method == XB.METHOD_AUTO:
            assert st.method == XB.METHOD_FUSED, "METHOD_AUTO should take the tensor cores at this size"
        for (gn, gp, gm), (rn, rp, rm) in zip(classes(got), classes(ref)):
            assert np.array_equal(gn, rn), ("NaN pattern", np.argwhere(gn != rn)[:5])
            assert np.array_equal(gp, rp), ("+Inf pattern", np.argwhere(gp != rp)[:5])
            assert np.array_equal(gm, rm), ("-Inf pattern", np.argwhere(gm != rm)[:5])
        fin = np.isfinite(ref) if not np.iscomplexobj(ref) else (np.isfinite(ref.real) & np.isfinite(ref.imag))
        assert fin.sum() > 0.9 * fin.size
        err = O.rel_frobenius(got[fin], ref[fin])
        assert err <= TOL[(st.method, dtk)], (accumulative, err)


def test_finite_inputs_need_no_fixup(xt, dev):
    """Without non-finite values the fix-up kernel returns at once: results
    are the tensor-core path's usual ones (bit-identical on repeat)."""
    dtk = O.R8
    L = rand_host(dtk, M * K, 41)
    R = rand_host(dtk, N * K, 42)
    outs = []
    for _ in range(2):
        dd, ld, rd = dev.put(np.zeros(M * N)), dev.put(L), dev.put(R)
        xt.tensor_contract(PATTERN, dtk, [M, N], dd.data_ptr(), [K, M], ld.data_ptr(), [K, N], rd.data_ptr(), 1.0,
                           plan=xt.make_plan(XB.METHOD_FUSED), stream=dev.stream())
        outs.append(dev.get(dd, np.float64, M * N))
    assert np.isfinite(outs[0]).all()
    assert np.array_equal(outs[0], outs[1])
    ref = (R.reshape(N, K) @ L.reshape(M, K).T).ravel()
    assert O.rel_frobenius(outs[0], ref) <= 1e-12
