"""sw_score_noalloc: scoring for callers that cannot allocate device memory.

Some callers must not call cudaMalloc where they score: a request path that
must not allocate once it runs (an allocation can block on the driver and
stall the requests behind it), or a plug-in whose host process has handed
all device memory to its own allocator.  The entry point takes device inputs
and a device output and keeps its scratch in a static device array inside
the library.  These tests compare it with the allocating search path and with
the oracle.  The file is collected last so that a failure here comes after
every other test has run."""
import numpy as np
import pytest

import oracle
from swhybrid_b200 import capi, param, synth

pytestmark = pytest.mark.gpu


def _upload(recs):
    import torch
    off = np.zeros(len(recs) + 1, dtype=np.uint64)
    off[1:] = np.cumsum([len(r) for r in recs])
    res = np.concatenate(recs).astype(np.uint8)
    dev = torch.device("cuda:0")
    return res, off, torch.from_numpy(res).to(dev), torch.from_numpy(off.astype(np.int64)).to(dev)


def test_noalloc_matches_search_on_two_calls_in_a_row():
    import torch
    rng = np.random.default_rng(31)
    q = synth.residues(rng, 700)                 # two query passes of 512 rows
    db = synth.small_db(8, 1500)
    db, _ = synth.plant_homologs(rng, db, q, 0.02)
    W = param.encode("W" * 3000)                 # exact above the 16-bit window (33000)
    recs = [db.record(i) for i in range(db.n)] + [W]
    res, off, d_res, d_off = _upload(recs)
    qW = np.concatenate([q, param.encode("W" * 3000)]).astype(np.uint8)

    params = capi.default_params(top_k=10)
    with capi.Context(0, params) as ctx:
        ctx.load_db(res, off)
        _, want = ctx.search(qW, want_scores=True)
    ref = oracle.search(qW, res, off, param.blosum62(), 12, 2, mode=1)
    np.testing.assert_array_equal(want, ref)

    dev = torch.device("cuda:0")
    d_q = torch.from_numpy(qW).to(dev)
    for call in range(2):
        d_out = torch.full((len(recs),), -7, dtype=torch.int32, device=dev)
        st = capi.score_noalloc(0, params, d_q.data_ptr(), len(qW), d_res.data_ptr(),
                                d_off.data_ptr(), len(recs), d_out.data_ptr())
        assert st == capi.SW_OK, f"call {call}: status {st}"
        got = d_out.cpu().numpy()
        np.testing.assert_array_equal(got, want, err_msg=f"call {call} vs sw_search")
        np.testing.assert_array_equal(got, ref, err_msg=f"call {call} vs oracle")
    assert want[-1] == oracle.gotoh(qW, W, param.blosum62()) > 32767


def test_noalloc_rejects_records_beyond_its_limit_and_scores_the_rest():
    import torch
    long_rec = synth.query(5, 9000)              # longer than the 8192-residue limit
    short_rec = synth.query(7, 400)
    _, _, d_res, d_off = _upload([long_rec, short_rec])
    q = synth.query(6, 100)
    d_q = torch.from_numpy(q).to("cuda:0")
    d_out = torch.full((2,), -7, dtype=torch.int32, device="cuda:0")
    st = capi.score_noalloc(0, capi.default_params(), d_q.data_ptr(), len(q), d_res.data_ptr(),
                            d_off.data_ptr(), 2, d_out.data_ptr())
    assert st == capi.SW_ERR_UNSUPPORTED
    want_short = oracle.gotoh(q, short_rec, param.blosum62())
    assert d_out.cpu().numpy().tolist() == [0, want_short]


def test_noalloc_reference_cap_on_a_caller_stream():
    import torch
    W = param.encode("W" * 6000)                 # W x W scores 11 per cell: 66000
    _, _, d_res, d_off = _upload([W])
    d_q = torch.from_numpy(W).to("cuda:0")
    stream = torch.cuda.Stream(device=0)
    exact = oracle.gotoh(W, W, param.blosum62())
    assert exact == 66000
    for cap, want in ((True, 65535), (False, exact)):
        d_out = torch.zeros(1, dtype=torch.int32, device="cuda:0")
        torch.cuda.synchronize()
        st = capi.score_noalloc(0, capi.default_params(reference_cap=cap), d_q.data_ptr(),
                                len(W), d_res.data_ptr(), d_off.data_ptr(), 1, d_out.data_ptr(),
                                stream.cuda_stream)
        assert st == capi.SW_OK
        assert int(d_out.cpu()[0]) == want, f"cap={cap}"
