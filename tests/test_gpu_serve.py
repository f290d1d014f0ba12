"""Request server (continuous batching over resident keys): every result equals
the raw proof the same witness gives alone through the plain path, whether the
request runs alone on an idle server or in a mix of circuits with requests of
several keys in flight, submitted from several host threads."""
import threading

import numpy as np
import pytest

import nkr_b200 as nk
import oracle as O

pytestmark = pytest.mark.gpu

SPECS = [("poseidon", 4, 1, 5), ("sql-aggregate", 8, 2, 4), ("matmul", 5, 0, 1), ("poseidon", 16, 2, 3)]


@pytest.fixture(scope="module")
def keyset(ctx):
    backends, wits = [], []
    for j, (kind, param, dens, nwit) in enumerate(SPECS):
        r1 = nk.generate(kind, param, dens, seed=500 + j)
        pk, _ = nk.setup(ctx, r1, O.random_fr(5, np.random.default_rng(600 + j)))
        be = nk.Backend(ctx)
        be.prepare(r1, pk)
        backends.append(be)
        wits.append([nk.generate(kind, param, dens, seed=700 + 10 * j + i).witness for i in range(nwit)])
    single = [[bytes(be.prove(w)) for w in ws] for be, ws in zip(backends, wits)]
    yield backends, wits, single
    for be in backends:
        be.free()


def test_alone_and_in_mix_equal_plain_proves(ctx, keyset):
    backends, wits, single = keyset
    sv = nk.Server(ctx, max_inflight=6, max_slots_per_key=3)
    ids = [sv.add_key(be) for be in backends]
    # alone: one request on an idle server
    rid = sv.submit(ids[1], wits[1][0])
    raw, lat, q = sv.wait(rid)
    assert bytes(raw) == single[1][0] and lat >= q >= 0
    # mix: all requests submitted back to back, interleaved across keys
    order = [(j, i) for i in range(5) for j in range(len(SPECS)) if i < len(wits[j])]
    rids = [(j, i, sv.submit(ids[j], wits[j][i])) for j, i in order]
    for j, i, r in rids:
        raw, lat, q = sv.wait(r)
        assert bytes(raw) == single[j][i], f"key {j} witness {i}"
    assert 1 <= sv.slots(ids[0]) <= 3
    sv.close()


def test_submitters_on_several_threads(ctx, keyset):
    backends, wits, single = keyset
    sv = nk.Server(ctx, max_inflight=8, max_slots_per_key=2)
    ids = [sv.add_key(be) for be in backends]
    errors = []

    def client(j):
        try:
            for rep in range(2):
                rs = [(i, sv.submit(ids[j], w)) for i, w in enumerate(wits[j])]
                for i, r in rs:
                    raw, _, _ = sv.wait(r)
                    if bytes(raw) != single[j][i]:
                        errors.append((j, i, rep))
        except Exception as e:  # surfaced below
            errors.append(repr(e))

    ts = [threading.Thread(target=client, args=(j,)) for j in range(len(SPECS))]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    sv.close()
    assert not errors, errors


def test_rejects_unknown_key_and_request(ctx, keyset):
    sv = nk.Server(ctx)
    with pytest.raises(nk.B200Error, match="unknown key"):
        sv.submit(3, keyset[1][0][0])
    with pytest.raises(nk.B200Error, match="unknown request"):
        sv.wait(12345)
    sv.close()


def test_large_key_proves_one_request_at_a_time(ctx):
    """A key of 2^19 rows fills the GPU alone: the server keeps it to one slot and
    queues its other requests in arrival order, while a small key beside it
    still takes several slots; every result equals the plain prove."""
    big = nk.generate("matmul", 64, 0, seed=900)          # 266,240 rows -> 2^19
    assert big.rows == 1 << 19
    small = nk.generate("poseidon", 4, 1, seed=901)
    bes = []
    for r1, seed in ((big, 902), (small, 903)):
        pk, _ = nk.setup(ctx, r1, O.random_fr(5, np.random.default_rng(seed)))
        be = nk.Backend(ctx)
        be.prepare(r1, pk)
        bes.append(be)
    small_wits = [nk.generate("poseidon", 4, 1, seed=910 + i).witness for i in range(4)]
    want_big = bytes(bes[0].prove(big.witness))
    want_small = [bytes(bes[1].prove(w)) for w in small_wits]
    sv = nk.Server(ctx, max_inflight=8, max_slots_per_key=4)
    kb, ks = sv.add_key(bes[0]), sv.add_key(bes[1])
    rb = [sv.submit(kb, big.witness) for _ in range(3)]
    rs = [sv.submit(ks, w) for w in small_wits]
    for r in rb:
        assert bytes(sv.wait(r)[0]) == want_big
    for r, w in zip(rs, want_small):
        assert bytes(sv.wait(r)[0]) == w
    assert sv.slots(kb) == 1
    assert 1 <= sv.slots(ks) <= 4
    sv.close()
    for be in bes:
        be.free()


def test_aged_requests_launch_at_top_priority_and_stay_exact(ctx, keyset):
    """With an ageing factor near zero every request that starts after its key's
    first completion is aged (launched into the slot's highest-priority stream,
    ordered after its witness upload); results still equal the plain proves and
    the server counts the aged launches."""
    backends, wits, single = keyset
    sv = nk.Server(ctx, max_inflight=6, max_slots_per_key=2)
    sv.set_ageing(1e-9)
    ids = [sv.add_key(be) for be in backends]
    for rep in range(3):
        rids = [(j, i, sv.submit(ids[j], wits[j][i])) for j in range(len(SPECS))
                for i in range(len(wits[j]))]
        for j, i, r in rids:
            assert bytes(sv.wait(r)[0]) == single[j][i], f"rep {rep} key {j} witness {i}"
    st = sv.stats()
    total = sum(len(w) for w in wits) * 3
    assert st["completed"] == total and st["failed"] == 0
    assert st["aged"] >= total - 2 * len(SPECS) * 2   # all but the first wave of each key
    with pytest.raises(nk.B200Error):
        sv.set_ageing(-1.0)
    sv.close()
