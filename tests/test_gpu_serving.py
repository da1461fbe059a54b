"""The request loop on the GPU: a seeded Poisson stream of uneven solves is
served with continuous batching in mixed precision, and every result is
compared with the same request solved alone.

Bars:
  * in the mix vs alone in a batch (same precision): bit-identical state;
  * mixed vs the plain FP64 stepper on the same request: max displacement
    error <= DISP_TOL relative to the largest FP64 displacement.
"""
import numpy as np
import pytest

from _common import rel
from enscdynamics_b200 import capi
from enscdynamics_b200 import serving as S
from enscdynamics_b200 import workloads as W

pytestmark = pytest.mark.gpu

DISP_TOL = 1e-5
FIELDS = ("x", "u", "v", "sigma", "qia", "eps_p")


def test_results_in_the_mix_equal_results_alone():
    reqs = W.serving_requests(12, rate=400.0, seed=21, ne_min=1000, ne_max=20000, steps=(200, 700))
    be = S.BatchBackend(budget_bytes=1 << 30, max_instances=8, max_elements=1 << 20, max_nodes=1 << 21,
                        fields=FIELDS)
    try:
        out = S.Server(be, min_quantum=32, prepare_workers=2, prepare_ahead=3).serve(reqs)
    finally:
        be.close()
    assert all(o.status == 0 for o in out)
    s = S.summarize(out)
    assert s["failed"] == 0 and s["solves_per_s"] > 0
    # the stream really overlapped: some request was admitted before another finished
    assert any(a.admitted < b.finished and b.admitted < a.finished
               for a in out for b in out if a.index != b.index)
    for o, r in zip(out, reqs):
        p = r.problem
        assert o.cycles == p.cycles
        with capi.Batch(max_instances=1, max_elements=1 << 20, max_nodes=1 << 21, budget_bytes=1 << 30,
                        precision=capi.MIXED) as b:
            slot = b.add(p.mesh.x0, p.mesh.conn, p.v0, material=p.material, controls=p.controls)
            b.set_bcs(slot, p.bc_code, p.bc_value)
            b.arm(slot, p.cycles)
            while b.sync() > 0:
                b.run(256)
            alone = b.download(slot)
        for k in FIELDS:
            assert np.array_equal(o.result[k], alone[k]), (o.index, k)
        with capi.Stepper(p.mesh.x0, p.mesh.conn, p.v0, material=p.material, controls=p.controls,
                          precision=capi.FP64) as st:
            st.set_bcs(p.bc_code, p.bc_value)
            st.step(p.cycles)
            ref = st.download()
        assert rel(o.result["u"], ref["u"]) <= DISP_TOL, (o.index, rel(o.result["u"], ref["u"]))
