"""Scoring matrices from text (sw_params_parse_matrix / sw_params_load_matrix,
the -m option): the built-in BLOSUM62 written out as text must parse back to
itself whatever the column order, case or extra letters; malformed texts are
refused.  Needs no GPU."""
import numpy as np
import pytest

from swhybrid_b200 import capi, param

ALPHA = param.ALPHABET


def to_text(m, letters, extra_star=True, lower=False):
    cols = list(letters) + (["*"] if extra_star else [])
    lines = ["# test matrix", "   " + " ".join(c.lower() if lower else c for c in cols)]
    for r in cols:
        vals = [(-4 if "*" in (r, c) else int(m[ALPHA.index(r), ALPHA.index(c)])) for c in cols]
        lines.append((r.lower() if lower else r) + " " + " ".join(f"{v:3d}" for v in vals))
    return "\n".join(lines) + "\n"


def test_blosum62_round_trip_any_order_and_case():
    m = param.blosum62()
    base = capi.load_matrix("blosum62")
    np.testing.assert_array_equal(base, m)
    np.testing.assert_array_equal(capi.load_matrix("BLOSUM62"), m)
    np.testing.assert_array_equal(capi.parse_matrix(to_text(m, ALPHA)), m)
    shuffled = "".join(np.random.default_rng(1).permutation(list(ALPHA)))
    np.testing.assert_array_equal(capi.parse_matrix(to_text(m, shuffled, lower=True)), m)


def test_missing_letters_score_zero_and_file_load(tmp_path):
    rng = np.random.default_rng(2)
    std = "ARNDCQEGHILKMFPSTWYV"
    r = rng.integers(-10, 16, size=(23, 23))
    r = np.triu(r) + np.triu(r, 1).T
    m = np.zeros((32, 32), dtype=np.int32)
    m[:23, :23] = r
    got = capi.parse_matrix(to_text(m, std, extra_star=False))
    want = np.zeros_like(m)
    idx = [ALPHA.index(c) for c in std]
    want[np.ix_(idx, idx)] = m[np.ix_(idx, idx)]
    np.testing.assert_array_equal(got, want)
    f = tmp_path / "m.txt"
    f.write_text(to_text(m, std))
    np.testing.assert_array_equal(capi.load_matrix(str(f)), want)


@pytest.mark.parametrize("text,status", [
    ("A R\nA 1 2\nR 3\n", 5),                 # short row
    ("A R\nA 1 2 3\nR 3 4\n", 5),             # long row
    ("A R\nA 1 200\nR 3 4\n", 1),             # out of range
    ("# only a comment\n", 5),                # no matrix
    ("A R\nA 1 2\nA 3 4\n", 5),               # repeated row
    ("AB R\nA 1 2\n", 5),                     # label not one letter
])
def test_malformed_texts(text, status):
    with pytest.raises(capi.SwError) as e:
        capi.parse_matrix(text)
    assert e.value.status == status


def test_unknown_name():
    with pytest.raises(capi.SwError):
        capi.load_matrix("no-such-matrix-or-file")
