"""Host logic of the serving loop's admission (no GPU): HBM bytes and sweep SMs.

A request is admitted when its bytes fit into the budget and at least
min(wanted CTAs, SMs / streams) SMs are free; it is granted min(wanted, free)
sweep CTAs, so the grants of running requests never exceed the SM count (their
cooperative sweeps fit on the GPU together)."""

import threading
import time

import numpy as np

from rapids_singlecell_b200.batched import HarmonyRequest, HarmonyServer, sweep_ctas_wanted


def _server(sms=148, streams=8, budget=1 << 40):
    srv = HarmonyServer.__new__(HarmonyServer)  # the admission state only: no device, no workers
    srv.budget, srv.in_use, srv.sms_in_use = budget, 0, 0
    srv.sms, srv.fair_ctas = sms, max(1, sms // streams)
    srv._cv = threading.Condition()
    return srv


def _req(n, block_proportion=0.05, n_clusters=4, precision="bf16"):
    return HarmonyRequest(np.zeros((n, 2), np.float32), np.zeros(n, np.int32), 1, None, np.ones(1),
                          dict(n_clusters=n_clusters, block_proportion=block_proportion), precision=precision)


def test_sweep_ctas_wanted():
    # one CTA per two tiles of a block (two tile streams per CTA up to 128 clusters)
    assert sweep_ctas_wanted(_req(1_000_000), 148) == 148    # 50,000-cell blocks: 391 tiles
    assert sweep_ctas_wanted(_req(20_000), 148) == 4          # 1,000-cell blocks: 8 tiles
    assert sweep_ctas_wanted(_req(20_000, n_clusters=200), 148) == 8  # one tile stream per CTA
    assert sweep_ctas_wanted(_req(100), 148) == 1
    assert sweep_ctas_wanted(_req(100_000, 1.0), 148) == 148
    # the plain paths have no cooperative sweep: no SMs asked for
    assert sweep_ctas_wanted(_req(20_000, precision="fp32"), 148) == 0
    assert sweep_ctas_wanted(_req(20_000, precision="fp64"), 148) == 0


def test_plain_requests_take_no_sms():
    srv = _server(sms=148, streams=8)
    assert srv._admit(10, 148) == 148   # a 16-bit request holds every SM
    assert srv._admit(10, 0) == 0       # a plain request is admitted all the same
    assert srv.sms_in_use == 148


def test_grants_stay_within_the_sms():
    srv = _server()
    g1 = srv._admit(10, 148)       # alone: the whole GPU
    assert g1 == 148 and srv.sms_in_use == 148
    got = []
    t = threading.Thread(target=lambda: got.append(srv._admit(10, 8)))
    t.start()
    time.sleep(0.2)
    assert not got                 # no SM free: waits
    srv._release(10, g1)
    t.join(5)
    assert got == [8] and srv.sms_in_use == 8
    g3 = srv._admit(10, 148)       # the rest, above the fair share of 18
    assert g3 == 140 and srv.sms_in_use == 148
    srv._release(10, 8)
    srv._release(10, g3)
    assert srv.sms_in_use == 0 and srv.in_use == 0


def test_large_request_waits_for_its_fair_share():
    srv = _server(sms=148, streams=8)   # fair share 18
    g = srv._admit(1, 140)              # 8 SMs left
    got = []
    t = threading.Thread(target=lambda: got.append(srv._admit(1, 148)))
    t.start()
    time.sleep(0.2)
    assert not got                      # 8 < 18: waits rather than run on 8 SMs
    srv._release(1, g)
    t.join(5)
    assert got == [148]
    srv._release(1, 148)


def test_bytes_are_admitted_by_budget():
    srv = _server(budget=100)
    srv._admit(60, 1)
    got = []
    t = threading.Thread(target=lambda: got.append(srv._admit(60, 1)))
    t.start()
    time.sleep(0.2)
    assert not got and srv.in_use == 60
    srv._release(60, 1)
    t.join(5)
    assert got == [1] and srv.in_use == 60
