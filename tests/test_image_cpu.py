"""DB image (sw_db_write_image / sw_fasta_to_image / sw_image_get_info): the
FASTA converter's records, titles and length order, read back from the file
with numpy, must equal a plain Python parse; damaged files must be refused.
Needs no GPU: these calls touch no device."""
import os
import struct

import numpy as np
import pytest

from swhybrid_b200 import capi

ALPHA = "ABCDEFGHIKLMNPQRSTVWXYZ"
HDR = struct.Struct("<8sII12Q")


def encode(text: str) -> np.ndarray:
    tab = {c: i for i, c in enumerate(ALPHA)}
    tab.update({c.lower(): i for i, c in enumerate(ALPHA)})
    tab["@"] = 23
    return np.array([tab.get(c, 24) for c in text if c not in " \t\r\n\v\f"], dtype=np.uint8)


def parse_fasta(text: str):
    titles, seqs = [], []
    for line in text.replace("\r\n", "\n").split("\n"):
        if line.startswith(">"):
            titles.append(line[1:].rstrip("\r"))
            seqs.append("")
        elif titles:
            seqs[-1] += line
    return titles, [encode(s) for s in seqs]


def read_image(path):
    raw = open(path, "rb").read()
    f = HDR.unpack_from(raw, 0)
    magic, version, hb, n, nres, o_off, o_res, o_toff, o_tit, tbytes, o_ord, fbytes, csum = f[:13]
    assert magic == b"SWB200DB" and version == 1 and hb == 128 and fbytes == len(raw)
    off = np.frombuffer(raw, np.uint64, n + 1, o_off)
    res = np.frombuffer(raw, np.uint8, nres, o_res)
    toff = np.frombuffer(raw, np.uint64, n + 1, o_toff)
    tit = raw[o_tit:o_tit + tbytes]
    order = np.frombuffer(raw, np.uint32, n, o_ord)
    recs = [res[off[i]:off[i + 1]] for i in range(n)]
    titles = [tit[toff[i]:toff[i + 1]].decode() for i in range(n)]
    return recs, titles, order


FASTA = (">sp|P1|first protein\r\nMKTAYIAKQR\r\nqisfvkshfs\r\n"
         ">second  with  spaces\nACDEFGHIKLMNPQRSTVWY\nBZX*JOU@\n\n"
         ">empty record\n"
         ">last\nMMMM\nMM")


def test_fasta_to_image_round_trip(tmp_path):
    fa = tmp_path / "db.fasta"
    fa.write_bytes(FASTA.encode())
    img = str(tmp_path / "db.swdb")
    info = capi.fasta_to_image(str(fa), img)
    titles, seqs = parse_fasta(FASTA)
    assert info["n_records"] == 4 and info["n_residues"] == sum(len(s) for s in seqs)
    recs, got_titles, order = read_image(img)
    assert got_titles == titles
    for a, b in zip(recs, seqs):
        np.testing.assert_array_equal(a, b)
    lens = [len(s) for s in seqs]
    assert list(order) == sorted(range(4), key=lambda i: (-lens[i], i))
    assert capi.image_info(img) == info


def test_write_image_and_damage(tmp_path):
    rng = np.random.default_rng(5)
    lens = rng.integers(0, 300, size=200)
    off = np.zeros(201, dtype=np.uint64)
    off[1:] = np.cumsum(lens)
    res = rng.integers(0, 25, size=int(off[-1])).astype(np.uint8)
    titles = [f"record {i}" for i in range(200)]
    img = str(tmp_path / "w.swdb")
    capi.write_image(img, res, off, titles)
    recs, got_titles, order = read_image(img)
    assert got_titles == titles
    for i in range(200):
        np.testing.assert_array_equal(recs[i], res[off[i]:off[i + 1]])
    assert list(order) == sorted(range(200), key=lambda i: (-int(lens[i]), i))
    assert not os.path.exists(img + ".tmp")
    good = open(img, "rb").read()
    # one flipped residue byte: only the checksum sees it
    bad = bytearray(good)
    bad[HDR.unpack_from(good, 0)[6] + 5] ^= 1
    open(img, "wb").write(bytes(bad))
    with pytest.raises(capi.SwError) as e:
        capi.image_info(img)
    assert e.value.status == 5 and "checksum" in str(e.value)
    capi.image_info(img, verify=False)
    # truncated, wrong magic
    open(img, "wb").write(good[:-64])
    with pytest.raises(capi.SwError) as e:
        capi.image_info(img)
    assert e.value.status == 5
    open(img, "wb").write(b"XXXXXXXX" + good[8:])
    with pytest.raises(capi.SwError) as e:
        capi.image_info(img)
    assert e.value.status == 5


def test_fasta_errors(tmp_path):
    fa = tmp_path / "bad.fasta"
    fa.write_text("MKT\n>x\nAAA\n")
    with pytest.raises(capi.SwError) as e:
        capi.fasta_to_image(str(fa), str(tmp_path / "bad.swdb"))
    assert e.value.status == 5
    empty = tmp_path / "empty.fasta"
    empty.write_text("")
    assert capi.fasta_to_image(str(empty), str(tmp_path / "e.swdb"))["n_records"] == 0
    with pytest.raises(capi.SwError):
        capi.fasta_to_image(str(tmp_path / "missing.fasta"), str(tmp_path / "m.swdb"))
