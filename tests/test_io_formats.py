"""Input formats on the host: the .2bit database reader (seq/twobit.rs) and gilist selection
(main.rs:1444-1470); no GPU needed."""
import numpy as np
import pytest

from rmblast_b200 import api, synth
from twobit_util import write_twobit


@pytest.mark.parametrize("big_endian", [False, True])
def test_twobit_matches_fasta_path(tmp_path, big_endian):
    """N runs are the only ambiguity a .2bit holds; both readers draw one CRandom number per N in
    position order from a generator seeded with the length, so they must agree base for base."""
    rng = np.random.default_rng(5)
    recs = []
    for i in range(6):
        s = bytearray(rng.choice(np.frombuffer(b"ACGT", dtype=np.uint8), size=int(rng.integers(50, 3000))).tobytes())
        for _ in range(int(rng.integers(0, 4))):
            a = int(rng.integers(0, len(s)))
            s[a:a + int(rng.integers(1, 80))] = b"N" * len(s[a:a + 80])
        if i == 2:
            s[10:40] = s[10:40].lower()  # soft mask: ignored
        recs.append((f"seq{i}", bytes(s[:len(s)])))
    path = tmp_path / "db.2bit"
    write_twobit(path, recs, big_endian)
    a = api.SubjectDb.from_twobit(path)
    b = api.SubjectDb.from_records([(n, s.upper()) for n, s in recs])
    assert a.ids == b.ids and a.deflines is None
    for pa, pb, ma, mb in zip(a.plus, b.plus, a.masks, b.masks):
        assert np.array_equal(pa, pb)
        assert (ma is None) == (mb is None)
        if ma is not None:
            assert np.array_equal(ma, mb)


def test_gilist_selection():
    _, db, _ = synth.workload("small", scale=0.1)
    sdb = api.SubjectDb.from_fasta(synth.to_fasta([f"gi|{i}" if i % 3 == 0 else n for i, (n, _) in enumerate(db)],
                                                  [s for _, s in db]))
    sel = sdb.select(["0", "gi|3", " " + sdb.ids[1] + " ", "", "nosuch"])
    assert sel.ids == ["gi|0", sdb.ids[1], "gi|3"]
    assert sel.deflines == [sdb.deflines[0], sdb.deflines[1], sdb.deflines[3]]
