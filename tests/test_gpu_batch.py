"""Batched stepping (ensc_batch_*): each instance of a batch must give the
results of the same solve run alone through ensc_create / ensc_step.

Bars:
  * FP64 and mixed: nodal x, u, v and element sigma, qia, eps_p bit-identical
    to the single-instance stepper of the same precision, and the same clock
    (time, dt_i, dt_i_1, cycles) -- both paths evaluate the same element and
    node bodies in the same order per element / node;
  * energy sums within ENERGY_REL of the single-instance sums (the batch sums
    per 32-element tile, the single stepper per thread block);
  * an instance's results do not depend on which other instances share the
    batch, on instances added or removed while it runs, or on the launch
    geometry and graph length the autotuner picks.
"""
import math

import numpy as np
import pytest

from _common import golden_names, load_golden, material_controls, run_len
from enscdynamics_b200 import capi
from enscdynamics_b200 import workloads as W

pytestmark = pytest.mark.gpu

ENERGY_REL = 1e-11
FIELDS = ("x", "u", "v", "sigma", "qia", "eps_p")


class Case:
    def __init__(self, name, x0, conn, v0, code, val, mat, ctl, cycles, end=math.inf):
        self.name, self.x0, self.conn, self.v0 = name, x0, conn, v0
        self.code, self.val, self.mat, self.ctl = code, val, mat, ctl
        self.cycles, self.end = cycles, end


def golden_case(name):
    g = load_golden(name)
    mat, ctl = material_controls(g["meta"])
    n, end = run_len(g)
    return Case(name, g["x0"], g["conn"], g["v0"], g["bc_code"], g["bc_value"], mat, ctl, n, end)


def sweep_case(i, cycles, plastic=True, ne_max=3000):
    p = W.sweep_instance(i, seed=3, ne_min=150, ne_max=ne_max, cycles=cycles)
    mat = p.material if plastic else W.M.Material(p.material.E, p.material.nu, p.material.rho)
    return Case(p.name, p.mesh.x0, p.mesh.conn, p.v0, p.bc_code, p.bc_value, mat, p.controls, cycles)


def single(case, precision, cycles=None):
    with capi.Stepper(case.x0, case.conn, case.v0, material=case.mat, controls=case.ctl,
                      precision=precision) as s:
        s.set_bcs(case.code, case.val)
        rep = s.step(case.cycles if cycles is None else cycles, case.end)
        return s.download(), rep, s.energy()


def make_batch(precision, **kw):
    args = dict(max_instances=16, max_elements=400000, max_nodes=500000, budget_bytes=2 << 30,
                precision=precision)
    args.update(kw)
    return capi.Batch(**args)


def add(b, case):
    slot = b.add(case.x0, case.conn, case.v0, material=case.mat, controls=case.ctl)
    b.set_bcs(slot, case.code, case.val)
    return slot


def drain(b, chunk=256, limit=10 ** 6):
    done = 0
    while b.sync() > 0:
        b.run(chunk)
        done += chunk
        assert done < limit
    return done


def assert_same(st, rep, en, ref, tag):
    st0, rep0, en0 = ref
    for k in FIELDS:
        assert np.array_equal(st[k], st0[k]), (tag, k, float(np.abs(st[k] - st0[k]).max()))
    for k in ("time", "dt_i", "dt_i_1", "cycles", "status"):
        assert rep[k] == rep0[k], (tag, k, rep[k], rep0[k])
    for k in ("kinetic", "internal", "hourglass", "viscous", "external", "kinetic0"):
        scale = max(abs(en0[k]), abs(en0["kinetic0"]), 1e-300)
        assert abs(en[k] - en0[k]) <= ENERGY_REL * scale, (tag, k, en[k], en0[k])


@pytest.mark.parametrize("precision", [capi.FP64, capi.MIXED])
def test_batch_matches_single_instances(precision):
    cases = [golden_case(n) for n in golden_names()]
    cases += [sweep_case(0, 170), sweep_case(1, 230, plastic=False), sweep_case(2, 95), sweep_case(5, 301)]
    refs = [single(c, precision) for c in cases]
    with make_batch(precision, max_instances=len(cases)) as b:
        slots = [add(b, c) for c in cases]
        for s, c in zip(slots, cases):
            b.arm(s, c.cycles, c.end)
        drain(b)
        for s, c, ref in zip(slots, cases, refs):
            assert_same(b.download(s), b.report(s), b.energy(s), ref, c.name)


@pytest.mark.parametrize("precision", [capi.FP64, capi.MIXED])
def test_instance_alone_equals_instance_in_mix(precision):
    target = sweep_case(4, 400)
    others = [sweep_case(i, 150 + 37 * i, ne_max=20000) for i in (6, 7, 8, 9, 10)]
    with make_batch(precision) as b:
        s = add(b, target)
        b.arm(s, target.cycles)
        drain(b)
        alone = (b.download(s), b.report(s), b.energy(s))
    with make_batch(precision) as b:
        ids = [add(b, c) for c in others[:2]]
        s = add(b, target)
        ids += [add(b, c) for c in others[2:]]
        for i, c in zip(ids, others):
            b.arm(i, c.cycles)
        b.arm(s, target.cycles)
        drain(b, chunk=64)
        mixed = (b.download(s), b.report(s), b.energy(s))
    assert_same(*mixed, alone, "mix")


def test_add_and_remove_while_others_run():
    """Instances join and leave between runs; the others are unaffected."""
    a, c, d = sweep_case(11, 300), sweep_case(12, 120), sweep_case(13, 200, plastic=False)
    refs = {k: single(v, capi.FP64) for k, v in (("a", a), ("d", d))}
    with make_batch(capi.FP64, graph_chunk=16) as b:
        sa = add(b, a)
        sc = add(b, c)
        b.arm(sa, 100)
        b.arm(sc, c.cycles)
        b.run(100)
        assert b.sync() == 1  # c is still running when it is removed
        b.remove(sc)
        assert b.instances == 1
        sd = add(b, d)  # may reuse the freed slot and its memory
        b.arm(sa, a.cycles - 100)
        b.arm(sd, d.cycles)
        drain(b, chunk=48)
        assert_same(b.download(sa), b.report(sa), b.energy(sa), refs["a"], "a")
        assert_same(b.download(sd), b.report(sd), b.energy(sd), refs["d"], "d")


def test_graph_length_does_not_change_results():
    cases = [sweep_case(14, 133), sweep_case(15, 77)]
    out = []
    for chunk in (0, 5, 64):
        with make_batch(capi.MIXED, graph_chunk=chunk) as b:
            ss = [add(b, c) for c in cases]
            for s, c in zip(ss, cases):
                b.arm(s, c.cycles)
            drain(b, chunk=50)
            out.append([b.download(s) for s in ss])
    for other in out[1:]:
        for r0, r1 in zip(out[0], other):
            for k in FIELDS:
                assert np.array_equal(r0[k], r1[k]), k


@pytest.mark.parametrize("precision", [capi.FP64, capi.MIXED])
def test_autotuner_tries_every_candidate_without_changing_results(precision):
    """A first run long enough for every launch candidate of the autotuner
    (grid sizes, graph lengths, both node-pass block sizes, 1 and 2 elements
    per thread in mixed precision) gives the single-instance results, and
    the choice it reports is one of them."""
    cases = [sweep_case(20, 900), sweep_case(21, 900, plastic=False)]
    refs = [single(c, precision) for c in cases]
    with make_batch(precision) as b:
        assert b.tuning == dict(mult_element=0, mult_node=0, graph_cycles=0, node_threads=0, elements_per_thread=0,
                                assembly=capi.ASSEMBLY_SLOT)
        ss = [add(b, c) for c in cases]
        for s, c in zip(ss, cases):
            b.arm(s, c.cycles)
        b.run(900)
        assert b.sync() == 0
        t = b.tuning
        assert t["mult_element"] in (1, 2) and t["mult_node"] in (1, 2)
        assert t["graph_cycles"] in (8, 32) and t["node_threads"] in (128, 256)
        assert t["elements_per_thread"] in ((1, 2) if precision == capi.MIXED else (1,))
        for s, c, ref in zip(ss, cases, refs):
            assert_same(b.download(s), b.report(s), b.energy(s), ref, c.name)


def test_budget_and_capacity_are_enforced():
    c = sweep_case(16, 10)
    with make_batch(capi.MIXED, budget_bytes=1 << 16) as b:
        with pytest.raises(capi.EnscError) as e:
            b.add(c.x0, c.conn, c.v0, material=c.mat, controls=c.ctl)
        assert e.value.code == -2
        assert b.instances == 0 and b.device_bytes == 0
    with make_batch(capi.MIXED, max_instances=1) as b:
        add(b, c)
        with pytest.raises(capi.EnscError) as e:
            b.add(c.x0, c.conn, c.v0, material=c.mat, controls=c.ctl)
        assert e.value.code == -2
        assert b.device_bytes > 0


def test_instance_reports_done_right_after_its_last_cycle():
    """A run that ends exactly on an instance's last cycle leaves it
    reported as finished by the next sync."""
    c = sweep_case(17, 100)
    with make_batch(capi.FP64, graph_chunk=10) as b:
        s = add(b, c)
        b.arm(s, 100)
        b.run(100)
        assert b.sync() == 0
        rep = b.report(s)
        assert rep["done"] == 1 and rep["cycles"] == 100


@pytest.mark.parametrize("precision", [capi.FP64, capi.MIXED])
def test_churn_with_short_runs_and_prepared_instances(precision):
    """The serving pattern: runs of 70 cycles (the autotuner then
    spreads its candidates over several runs), instances prepared on the
    host beforehand (ensc_batch_prepare / ensc_batch_add_prepared), and
    instances removed and added between runs, slots reused before the tables
    are rewritten.  Every instance still ends with its single-instance
    results and energies."""
    cases = [sweep_case(40 + i, 260 + 45 * i, plastic=i % 2 == 0) for i in range(6)]
    refs = [single(c, precision) for c in cases]
    got = {}
    with make_batch(precision, max_instances=4) as b:
        todo = list(range(len(cases)))
        live = {}

        def admit():
            while todo and len(live) < 3:
                i = todo.pop(0)
                c = cases[i]
                pr = capi.Prepared(c.x0, c.conn, c.v0, material=c.mat, controls=c.ctl, precision=precision)
                s = b.add_prepared(pr)
                pr.close()
                b.set_bcs(s, c.code, c.val)
                b.arm(s, c.cycles)
                live[s] = i
        admit()
        runs = 0
        while live:
            b.run(70)
            runs += 1
            b.sync()
            for s in list(live):
                if b.report(s)["done"]:
                    i = live.pop(s)
                    got[i] = (b.download(s), b.report(s), b.energy(s))
                    b.remove(s)
            admit()
            assert runs < 1000
        t = b.tuning
        assert t["graph_cycles"] in (8, 32)
    for i, c in enumerate(cases):
        assert_same(*got[i], refs[i], c.name)


@pytest.mark.parametrize("assembly", [capi.ASSEMBLY_SLOT, capi.ASSEMBLY_PATCH])
def test_mixed_batch_matches_single_under_each_assembly(assembly):
    cases = [sweep_case(50, 260), sweep_case(51, 190, plastic=False), sweep_case(52, 330)]
    refs = []
    for c in cases:
        with capi.Stepper(c.x0, c.conn, c.v0, material=c.mat, controls=c.ctl, precision=capi.MIXED,
                          assembly=assembly) as s:
            s.set_bcs(c.code, c.val)
            rep = s.step(c.cycles)
            refs.append((s.download(), rep, s.energy()))
    with make_batch(capi.MIXED, assembly=assembly) as b:
        ss = [add(b, c) for c in cases]
        for s, c in zip(ss, cases):
            b.arm(s, c.cycles)
        drain(b)
        for s, c, ref in zip(ss, cases, refs):
            assert_same(b.download(s), b.report(s), b.energy(s), ref, c.name)


def test_prepared_instance_must_match_the_batch():
    c = sweep_case(60, 10)
    with make_batch(capi.MIXED) as b:
        for prec, asm in ((capi.FP64, capi.ASSEMBLY_AUTO), (capi.MIXED, capi.ASSEMBLY_PATCH)):
            pr = capi.Prepared(c.x0, c.conn, c.v0, material=c.mat, controls=c.ctl, precision=prec, assembly=asm)
            with pytest.raises(capi.EnscError, match="ENSC_ERR_ARG"):
                b.add_prepared(pr)
            pr.close()
        assert b.instances == 0


@pytest.mark.parametrize("precision", [capi.FP64, capi.MIXED])
def test_prepared_instance_outlives_its_mesh_arrays(precision):
    """A prepared instance holds everything the device part copies: its mesh
    arrays can be overwritten and freed before ensc_batch_add_prepared, and
    the instance still runs as one added directly."""
    c = sweep_case(7, 60)
    x0, conn, v0 = c.x0.copy(), c.conn.copy(), c.v0.copy()
    pr = capi.Prepared(x0, conn, v0, material=c.mat, controls=c.ctl, precision=precision)
    x0[:] = np.nan
    v0[:] = np.nan
    conn[:] = 0
    del x0, conn, v0
    with make_batch(precision) as b:
        s = b.add_prepared(pr)
        pr.close()
        b.set_bcs(s, c.code, c.val)
        t = add(b, c)
        for slot in (s, t):
            b.arm(slot, c.cycles)
        drain(b)
        got, ref = b.download(s), b.download(t)
        for k in ("x", "u", "v", "sigma"):
            assert np.array_equal(got[k], ref[k]), k


@pytest.mark.parametrize("precision", [capi.FP64, capi.MIXED])
def test_instance_added_while_cycles_run(precision):
    """An instance added (upload, init pass, boundary conditions, arming on
    the batch's admission stream) while cycles enqueued for the others are
    still running joins at the next run, and every result equals the same
    instance alone."""
    first, late = sweep_case(3, 2000, ne_max=20000), sweep_case(11, 400)
    alone = {}
    for c in (first, late):
        with make_batch(precision) as b:
            s = add(b, c)
            b.arm(s, c.cycles)
            drain(b)
            alone[c.name] = (b.download(s), b.report(s), b.energy(s))
    with make_batch(precision) as b:
        a = add(b, first)
        b.arm(a, first.cycles)
        b.run(700)  # the launch geometry is tuned during the first runs
        b.sync()
        b.run(512)  # enqueued; the add below overlaps these cycles
        s = add(b, late)
        b.arm(s, late.cycles)
        drain(b)
        assert_same(b.download(a), b.report(a), b.energy(a), alone[first.name], first.name)
        assert_same(b.download(s), b.report(s), b.energy(s), alone[late.name], late.name)
