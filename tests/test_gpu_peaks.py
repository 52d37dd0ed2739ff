"""The tensor-core throughput probes (tb_peak_measure) that give the
contraction rooflines: each runs, reports a rate within the physically
possible range of a B200 (dense INT8 and BF16 tcgen05, FP64 DMMA), and INT8
runs at about twice the BF16 rate (twice the operations per MMA, same issue
rate)."""
import pytest

import exatensor_b200 as XB

pytestmark = pytest.mark.gpu


def test_peak_probes(xt, dev):
    i8, ms = xt.peak_measure(XB.PEAK_I8, 100000, dev.stream())
    bf, _ = xt.peak_measure(XB.PEAK_BF16, 100000, dev.stream())
    f64, _ = xt.peak_measure(XB.PEAK_F64, 20000, dev.stream())
    assert ms > 0
    assert 1.0e15 < i8 < 5.5e15, i8
    assert 0.5e15 < bf < 2.8e15, bf
    assert 1.0e13 < f64 < 1.0e14, f64
    assert 1.6 < i8 / bf < 2.4, (i8, bf)
    xt.device_check(dev.stream())


def test_peak_probe_rejects_bad_arguments(xt):
    with pytest.raises(XB.TBError):
        xt.peak_measure(99, 10)
    with pytest.raises(XB.TBError):
        xt.peak_measure(XB.PEAK_I8, 0)
