"""analysis (run.F90:238-388) on the GPU against the oracle: vorticity and
swirl maxima, the centroid sums and ratios, the centroid speeds from a second
call, the ghost-row side effect on q1..q3, and the analysis.dat line."""
import numpy as np
import pytest

from tests.parity_util import make_pair

pytestmark = pytest.mark.gpu


def test_analysis_matches_oracle(tmp_path):
    from vring_b200.synthetic import ring_fields
    nth, nr, nz = 16, 48, 96
    orc, gpu = make_pair(nth, nr, nz, dt=2e-3, wth="modified")
    for n, a in zip(("q1", "q2", "q3"), ring_fields(nth, nr, nz, 4.0, 12.0, noise=1e-3, seed=2)):
        orc.field(n)[...] = a
        gpu.set(n, a)
    # a swirl component so both centroids are defined
    rm = (np.arange(nr + 3) - 0.5) * (4.0 / nr)
    q1 = orc.field("q1")
    q1 += 0.3 * np.exp(-((rm[None, :, None] - 1.0) ** 2) / 0.1)
    gpu.set("q1", q1)
    path = tmp_path / "analysis.dat"
    outs = []
    for call in range(2):
        o_ref = orc.analysis(5)
        o_gpu = gpu.analysis(5, path=path)
        outs.append(o_gpu)
        for n in ("q1", "q2", "q3"):
            g = gpu.get(n)
            # ghost row 0 is row 1 on iz = 1..nz after the call (run.F90:305-307)
            np.testing.assert_array_equal(g[:, 0, 1:nz + 1], g[:, 1, 1:nz + 1])
            r = orc.field(n)
            assert np.abs(g - r).max() <= 1e-10 * np.abs(r).max(), n
        if call == 0:
            np.testing.assert_allclose(o_gpu[:11], o_ref[:11], rtol=1e-12)
            assert np.isnan(o_ref[11]) and np.isnan(o_gpu[11])        # 0/0 at the first call
        else:
            np.testing.assert_allclose(o_gpu, o_ref, rtol=1e-8)
        gpu.iterate(5)
        orc.iterate(5)
    lines = path.read_text().splitlines()
    assert len(lines) == 1 or len(lines) == 2     # rewound at nstep 1, appended otherwise
    last = lines[-1]
    assert len(last) == 5 + 13 * 16
    vals = [float(last[5 + 16 * i:5 + 16 * (i + 1)].replace("-0", "-0").strip() or "nan")
            for i in range(13)]
    np.testing.assert_allclose(vals[:11], outs[-1][:11], rtol=1e-7)
