"""sw_score_noalloc: scoring for callers that cannot allocate device memory
(a request path that must not allocate, a host process whose device memory
belongs to another allocator, work enqueued during stream capture).  Its
scratch is a static device array inside the library.  This file is collected
last so that a failure here comes after every other test has run."""
import numpy as np
import pytest

import oracle
from swhybrid_b200 import capi, param, synth

pytestmark = pytest.mark.gpu


def test_noalloc_matches_search_on_two_calls_in_a_row():
    import torch
    rng = np.random.default_rng(31)
    q = synth.residues(rng, 700)                 # two query passes of 512 rows
    db = synth.small_db(8, 1500)
    db, _ = synth.plant_homologs(rng, db, q, 0.02)
    W = param.encode("W" * 3000)                 # exact above the 16-bit window (33000)
    recs = [db.record(i) for i in range(db.n)] + [W]
    off = np.zeros(len(recs) + 1, dtype=np.uint64)
    off[1:] = np.cumsum([len(r) for r in recs])
    res = np.concatenate(recs).astype(np.uint8)
    qW = np.concatenate([q, param.encode("W" * 3000)]).astype(np.uint8)

    params = capi.default_params(top_k=10)
    with capi.Context(0, params) as ctx:
        ctx.load_db(res, off)
        _, want = ctx.search(qW, want_scores=True)

    dev = torch.device("cuda:0")
    d_q = torch.from_numpy(qW).to(dev)
    d_res = torch.from_numpy(res).to(dev)
    d_off = torch.from_numpy(off.astype(np.int64)).to(dev)
    for call in range(2):
        d_out = torch.full((len(recs),), -7, dtype=torch.int32, device=dev)
        st = capi.score_noalloc(0, params, d_q.data_ptr(), len(qW), d_res.data_ptr(),
                                d_off.data_ptr(), len(recs), d_out.data_ptr())
        assert st == capi.SW_OK, f"call {call}: status {st}"
        np.testing.assert_array_equal(d_out.cpu().numpy(), want, err_msg=f"call {call}")
    assert want[-1] == oracle.gotoh(qW, W, param.blosum62()) > 32767


def test_noalloc_rejects_records_beyond_its_limit():
    import torch
    dev = torch.device("cuda:0")
    rec = synth.query(5, 9000)                   # longer than the 8192-residue limit
    d_res = torch.from_numpy(rec).to(dev)
    d_off = torch.tensor([0, len(rec)], dtype=torch.int64, device=dev)
    d_q = torch.from_numpy(synth.query(6, 100)).to(dev)
    d_out = torch.zeros(1, dtype=torch.int32, device=dev)
    st = capi.score_noalloc(0, capi.default_params(), d_q.data_ptr(), 100, d_res.data_ptr(),
                            d_off.data_ptr(), 1, d_out.data_ptr())
    assert st == 6          # SW_ERR_UNSUPPORTED
