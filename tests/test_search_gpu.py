"""GPU parity of the plain search path, through the C ABI (libswb200.so).

Every record's score must equal the reference's (its own AVX2 int8 kernel +
RecalcWorker int16 pass, as stored in tests/golden/ by make_golden.py, or the
oracle restatement pinned to those vectors), bit for bit; top-k must equal the
oracle's under the stated tie order (score descending, record index
ascending)."""
import os

import numpy as np
import pytest

import oracle
from swhybrid_b200 import capi, param, synth

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
M = param.blosum62()


def load(name):
    z = np.load(os.path.join(GOLD, name + ".npz"))
    qo = z["qoffsets"].astype(np.int64)
    queries = [z["queries"][qo[i]:qo[i + 1]] for i in range(len(qo) - 1)]
    return z["residues"], z["offsets"], queries, z["scores"]


@pytest.fixture(scope="module")
def ctx():
    c = capi.Context(0, capi.default_params(top_k=10))
    yield c
    c.close()


def check_topk(hits, scores, k=10):
    sc, idx = oracle.topk(scores, k)
    assert [h[0] for h in hits] == sc.tolist()
    assert [h[1] for h in hits] == idx.tolist()


@pytest.mark.parametrize("name", ["edge", "homolog", "saturation"])
def test_golden_sets_bit_exact(ctx, name):
    res, off, queries, gold = load(name)
    ctx.load_db(res, off)
    for qi, q in enumerate(queries):
        hits, scores = ctx.search(q, want_scores=True)
        np.testing.assert_array_equal(scores, gold[qi], err_msg=f"{name} query {qi} len {len(q)}")
        check_topk(hits, gold[qi])


def test_small20k_query375_bit_exact(ctx):
    z = np.load(os.path.join(GOLD, "small20k_q375.npz"))
    db = synth.small_db(1, 20_000)
    q = synth.query(375, 375)
    ctx.load_db(db.residues, db.offsets)
    hits, scores = ctx.search(q, want_scores=True)
    np.testing.assert_array_equal(scores, z["scores"])
    check_topk(hits, z["scores"])


def all_shapes(ctx):
    """Every compiled (group width, rows per thread) shape."""
    return capi.shapes()


def test_every_kernel_shape_bit_exact(ctx):
    res, off, queries, gold = load("homolog")
    ctx.load_db(res, off)
    try:
        ran = 0
        for T, R in all_shapes(ctx):
            ctx.set_kernel_config((T, R, T, R, 0))
            for qi in (0, 1):
                try:
                    _, scores = ctx.search(queries[qi], want_scores=True)
                except capi.SwError as e:
                    # a profile that does not fit shared memory is refused, not run
                    assert e.status == 6, str(e)
                    continue
                ran += 1
                np.testing.assert_array_equal(scores, gold[qi], err_msg=f"shape {T}x{R} q{qi}")
        assert ran >= 90
    finally:
        ctx.set_kernel_config(None)


def test_cutover_split_bit_exact(ctx):
    res, off, queries, gold = load("homolog")
    ctx.load_db(res, off)
    try:
        for cfg in [(32, 32, 8, 16, 400), (16, 24, 4, 32, 1000), (8, 64, 4, 10, 200), (32, 6, 16, 12, 1500)]:
            ctx.set_kernel_config(cfg)
            for qi in (0, 1):
                _, scores = ctx.search(queries[qi], want_scores=True)
                np.testing.assert_array_equal(scores, gold[qi], err_msg=f"config {cfg}")
    finally:
        ctx.set_kernel_config(None)


def test_long_pairs_near_the_plain_step_bounds(ctx):
    """The long-pair kernel runs unguarded column steps only while every lane
    of a warp is inside its pair (steps 63 .. ncols - 2); pairs of 40..140
    columns (those above 60 in the long kernel) put the first and last plain
    steps at every offset from a barrier, with one to three pipelined passes,
    against the oracle."""
    rng = np.random.default_rng(43)
    lens = rng.integers(40, 141, size=600)
    db = synth.db_from_lengths(rng, lens)
    qs = [synth.residues(rng, L) for L in (200, 700)]
    db, _ = synth.plant_homologs(rng, db, qs[1], 0.03)
    wants = [oracle.search(q, db.residues, db.offsets, M, 12, 2) for q in qs]
    ctx.load_db(db.residues, db.offsets)
    try:
        for rows in (8, 16, 24):
            for q, want in zip(qs, wants):
                ctx.set_kernel_config((32, rows, 8, 12, 60))
                _, scores = ctx.search(q, want_scores=True)
                np.testing.assert_array_equal(scores, want, err_msg=f"R={rows} qlen={len(q)}")
                assert ctx.run_stats().long_ms > 0
    finally:
        ctx.set_kernel_config(None)


def test_streamed_segments_short_and_empty_records(ctx):
    """The plain kernel's groups stream from pass to pass and pair to pair
    without draining the wavefront.  Records of 0..80 residues (pairs shorter
    than the 2T+2 steps a pass that the next one depends on is padded to, runs
    of empty records) under a query of several passes for every group width,
    and DBs with fewer pairs than thread groups, against the oracle."""
    rng = np.random.default_rng(41)
    q = synth.residues(rng, 700)
    lens = rng.integers(0, 81, size=900)
    lens[::37] = 0
    lens[100:106] = 0
    big = synth.db_from_lengths(rng, lens)
    big, _ = synth.plant_homologs(rng, big, q, 0.02)
    dbs = [big] + [synth.db_from_lengths(rng, np.array(l)) for l in ([5], [0, 70], [66, 1, 2], [700, 3, 0, 64, 65])]
    wants = [oracle.search(q, d.residues, d.offsets, M, 12, 2) for d in dbs]
    try:
        for d, want in zip(dbs, wants):
            ctx.load_db(d.residues, d.offsets)
            for T, R in [(4, 8), (8, 12), (16, 6), (16, 48), (32, 4), (32, 10), (32, 40)]:
                ctx.set_kernel_config((T, R, T, R, 0))
                _, scores = ctx.search(q, want_scores=True)
                np.testing.assert_array_equal(scores, want, err_msg=f"{T}x{R} n={d.n}")
    finally:
        ctx.set_kernel_config(None)


def test_int16_threshold_and_int32_pass():
    """Scores around the 16-bit overflow threshold and above 65535: the 32-bit
    re-score must be exact; the reference cap reports 65535."""
    res, off, queries, gold = load("saturation")
    with capi.Context(0, capi.default_params(reference_cap=False)) as c:
        c.load_db(res, off)
        L = np.diff(off.astype(np.int64))
        for q in queries:
            _, scores = c.search(q, want_scores=True)
            np.testing.assert_array_equal(scores, 11 * np.minimum(L, len(q)))
        st = c.run_stats()
        assert st.rescored > 0


def test_long_records_and_many_passes(ctx):
    """Records up to 12,000 residues and a 3,000-residue query (several
    passes for every shape) against the oracle."""
    rng = np.random.default_rng(21)
    q = synth.residues(rng, 3000)
    lens = np.concatenate([rng.integers(8000, 12000, size=6), rng.integers(1, 400, size=50)])
    db = synth.db_from_lengths(rng, lens)
    db, _ = synth.plant_homologs(rng, db, q, 0.05)
    want = oracle.search(q, db.residues, db.offsets, M, 12, 2, mode=1)
    ctx.load_db(db.residues, db.offsets)
    hits, scores = ctx.search(q, want_scores=True)
    np.testing.assert_array_equal(scores, want)
    check_topk(hits, want)


# compiled long-pair row counts, plus 48 (not compiled: the automatic choice)
LONG_ROWS = (8, 16, 24, 32, 48, 64)


@pytest.fixture(scope="module")
def long_case():
    """Records of 1,600..9,000 residues (long pairs) among short ones, with
    planted homologs (scores far above the int8 range), and queries whose
    pass count runs from 1 to the 8-warp maximum of the long-pair kernel."""
    rng = np.random.default_rng(31)
    lens = np.concatenate([rng.integers(1600, 9000, size=120), rng.integers(5, 600, size=900)])
    lens = lens[rng.permutation(len(lens))]
    db = synth.db_from_lengths(rng, lens)
    queries = [synth.residues(rng, L) for L in (100, 700, 2100, 4097, 8000)]
    db, _ = synth.plant_homologs(rng, db, queries[2], 0.02)
    want = [oracle.search(q, db.residues, db.offsets, M, 12, 2) for q in queries]
    return db, queries, want


@pytest.mark.parametrize("rows", LONG_ROWS)
def test_long_pair_pipeline_every_row_count(ctx, long_case, rows):
    """Pairs above the cut-over go to the long-pair kernel (one warp per query
    pass, passes pipelined through shared memory, several pipelines per
    block); every row count and pass count must give the oracle's scores."""
    db, queries, want = long_case
    ctx.load_db(db.residues, db.offsets)
    try:
        ran = 0
        for q, w in zip(queries, want):
            if len(q) > 8 * 32 * rows:
                continue
            ctx.set_kernel_config((32, rows, 16, 16, 1500))
            hits, scores = ctx.search(q, want_scores=True)
            np.testing.assert_array_equal(scores, w, err_msg=f"R={rows} qlen={len(q)}")
            check_topk(hits, w)
            st = ctx.run_stats()
            assert st.long_ms > 0 and st.bulk_ms > 0
            assert st.used.cutover == 1500
            ran += 1
        assert ran >= 2
    finally:
        ctx.set_kernel_config(None)


def test_automatic_cutover_on_a_long_tailed_db(ctx, long_case):
    """Without a configured cut-over, a DB whose longest pairs dominate gets
    one automatically, and the scores stay exact."""
    db, queries, want = long_case
    ctx.load_db(db.residues, db.offsets)
    ctx.set_kernel_config((16, 16, 16, 16, 0))
    try:
        _, scores = ctx.search(queries[1], want_scores=True)
        np.testing.assert_array_equal(scores, want[1])
        st = ctx.run_stats()
        assert st.used.cutover >= 1024 and st.long_ms > 0
    finally:
        ctx.set_kernel_config(None)


def test_segmented_query_and_refused_search(ctx, long_case):
    """With a long-pair split configured, a query whose profile does not fit
    one block of the bulk shape (4,097 rows for 4x32) is scored in row
    segments by consecutive bulk launches beside the long-pair launch; and a
    search refused before launching (a bad residue code) leaves nothing in
    flight, so the next search is exact."""
    db, lq, lwant = long_case
    ctx.load_db(db.residues, db.offsets)
    try:
        ctx.set_kernel_config((32, 16, 4, 32, 1500))
        _, scores = ctx.search(lq[3], want_scores=True)
        np.testing.assert_array_equal(scores, lwant[3])
        bad = lq[1].copy()
        bad[5] = 25
        with pytest.raises(capi.SwError) as e:
            ctx.search(bad)
        assert e.value.status == 1
        _, scores = ctx.search(lq[0], want_scores=True)
        np.testing.assert_array_equal(scores, lwant[0])
    finally:
        ctx.set_kernel_config(None)


def test_other_gap_costs_match_oracle():
    rng = np.random.default_rng(22)
    db = synth.small_db(5, 800)
    q = synth.residues(rng, 300)
    for go, ge in [(11, 1), (5, 3), (0, 1)]:
        with capi.Context(0, capi.default_params(gap_open=go, gap_extend=ge, reference_cap=False)) as c:
            c.load_db(db.residues, db.offsets)
            _, scores = c.search(q, want_scores=True)
        want = oracle.search(q, db.residues, db.offsets, M, go + ge, ge, mode=0)
        np.testing.assert_array_equal(scores, want, err_msg=f"gaps {go}/{ge}")


def test_deterministic_and_order_invariant(ctx):
    db = synth.small_db(7, 3000)
    q = synth.query(8, 500)
    ctx.load_db(db.residues, db.offsets)
    h1, s1 = ctx.search(q, want_scores=True)
    h2, s2 = ctx.search(q, want_scores=True)
    assert h1 == h2
    np.testing.assert_array_equal(s1, s2)
    perm = np.random.default_rng(1).permutation(db.n)
    sub = db.subset(perm)
    ctx.load_db(sub.residues, sub.offsets)
    _, s3 = ctx.search(q, want_scores=True)
    np.testing.assert_array_equal(s3, s1[perm])


def test_empty_inputs(ctx):
    res = np.zeros(0, dtype=np.uint8)
    ctx.load_db(res, np.zeros(4, dtype=np.uint64))        # three empty records
    hits, scores = ctx.search(synth.query(1, 50), want_scores=True)
    assert hits == [] and scores.tolist() == [0, 0, 0]
    db = synth.small_db(2, 100)
    ctx.load_db(db.residues, db.offsets)
    hits, scores = ctx.search(np.zeros(0, dtype=np.uint8), want_scores=True)
    assert hits == [] and not scores.any()


def test_bad_codes_rejected(ctx):
    db = synth.small_db(2, 100)
    ctx.load_db(db.residues, db.offsets)
    bad = synth.query(1, 50)
    bad[3] = 40
    with pytest.raises(capi.SwError) as e:
        ctx.search(bad)
    assert e.value.status == 1


def test_query_longer_than_the_bound_refused(ctx):
    """Queries of more than 2^24 residues are refused before any device work
    (the plain, the resident and the batched entry points), and the context
    keeps working."""
    import torch
    db = synth.small_db(2, 100)
    ctx.load_db(db.residues, db.offsets)
    big = np.zeros((1 << 24) + 1, dtype=np.uint8)
    with pytest.raises(capi.SwError) as e:
        ctx.search(big)
    assert e.value.status == 6
    d_big = torch.from_numpy(big).cuda()
    with pytest.raises(capi.SwError) as e:
        ctx.search_device(d_big.data_ptr(), big.size)
    assert e.value.status == 6
    with pytest.raises(capi.SwError) as e:
        ctx.search_batch([synth.query(1, 50), big])
    assert e.value.status == 6
    q = synth.query(1, 50)
    hits, scores = ctx.search(q, want_scores=True)
    want = oracle.search(q, db.residues, db.offsets, M, 12, 2, mode=1)
    np.testing.assert_array_equal(scores, want)
