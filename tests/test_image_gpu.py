"""A DB loaded from its image (sw_db_load_image) searches exactly like the
same records loaded from memory, gives each hit's title, and a damaged image
is refused before anything reaches the device."""
import numpy as np
import pytest

from swhybrid_b200 import capi, synth

pytestmark = pytest.mark.gpu


def test_image_search_equals_memory_and_titles(tmp_path):
    rng = np.random.default_rng(81)
    db = synth.small_db(82, 3000)
    q = synth.residues(rng, 400)
    db, planted = synth.plant_homologs(rng, db, q, 0.01)
    titles = [f"seq{i} synthetic record of {int(db.offsets[i + 1] - db.offsets[i])} residues"
              for i in range(db.n)]
    img = str(tmp_path / "db.swdb")
    capi.write_image(img, db.residues, db.offsets, titles)
    with capi.Context(0) as a, capi.Context(0) as b:
        a.load_db(db.residues, db.offsets)
        b.load_image(img)
        ha, sa = a.search(q, want_scores=True)
        hb, sb = b.search(q, want_scores=True)
        np.testing.assert_array_equal(sa, sb)
        assert ha == hb
        assert [b.title(i) for (_, i) in hb] == [titles[i] for (_, i) in hb]
        with pytest.raises(capi.SwError) as e:
            a.title(0)                       # loaded from memory: no titles
        assert e.value.status == 4


def test_damaged_image_refused(tmp_path):
    db = synth.small_db(83, 500)
    img = str(tmp_path / "d.swdb")
    capi.write_image(img, db.residues, db.offsets)
    raw = bytearray(open(img, "rb").read())
    raw[-100] ^= 0x40
    open(img, "wb").write(bytes(raw))
    with capi.Context(0) as c:
        with pytest.raises(capi.SwError) as e:
            c.load_image(img)
        assert e.value.status == 5
