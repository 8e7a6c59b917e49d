"""EVP influence files (the PREP -> MAIN record): exact bytes of the
big-endian Fortran unformatted record, gfortran subrecords, the optional OAC
plane MAIN reads, and a round trip of PRE1 influence data.  Host code only."""
import numpy as np
import pytest

from musoc_solver_b200 import evp, native, problems as P


def _arrays(i2=7, j2=5, nb0=3, seed=0):
    g = np.random.default_rng(seed)
    planes = [g.standard_normal((j2, i2)).astype(np.float32) for _ in range(6)]
    rinv = g.standard_normal((nb0, i2, i2))
    rinv1 = g.standard_normal((nb0 - 1, i2, i2))
    ie = np.arange(2, 2 + 2 * nb0, 2, dtype=np.int32)
    return planes, rinv, rinv1, ie


def _expected_payload(planes, rinv, rinv1, ie, with_oac):
    parts = [a.astype(">f4").tobytes() for a in planes[:5]]
    if with_oac:
        parts.append(planes[5].astype(">f4").tobytes())
    parts += [rinv.astype(">f8").tobytes(), rinv1.astype(">f8").tobytes(), ie.astype(">i4").tobytes()]
    return b"".join(parts)


@pytest.mark.parametrize("with_oac", [False, True])
def test_record_bytes_and_round_trip(tmp_path, with_oac):
    native.lib()
    planes, rinv, rinv1, ie = _arrays()
    f = tmp_path / "EVP"
    evp.write(f, *planes[:5], rinv, rinv1, ie, oac=planes[5] if with_oac else None)
    payload = _expected_payload(planes, rinv, rinv1, ie, with_oac)
    marker = np.array([len(payload)], ">i4").tobytes()
    assert f.read_bytes() == marker + payload + marker
    r = evp.read(f, 7, 5, rinv.shape, rinv1.shape, len(ie))
    for k, a in zip(("al", "ar", "ab", "at", "ac"), planes):
        assert np.array_equal(r[k], a)
    assert np.array_equal(r["rinv"], rinv) and np.array_equal(r["rinv1"], rinv1)
    assert np.array_equal(r["ie"], ie)
    assert (r["oac"] is not None) == with_oac
    if with_oac:
        assert np.array_equal(r["oac"], planes[5])


def test_subrecords(tmp_path):
    planes, rinv, rinv1, ie = _arrays(seed=1)
    f = tmp_path / "EVP"
    evp.write(f, *planes[:5], rinv, rinv1, ie, max_subrecord=100)
    payload = _expected_payload(planes, rinv, rinv1, ie, False)
    raw = f.read_bytes()
    # walk the subrecords: negative leading marker = more follow, negative
    # trailing marker = continuation of an earlier subrecord
    pos, got, k = 0, b"", 0
    while True:
        lead = int(np.frombuffer(raw[pos:pos + 4], ">i4")[0])
        n = abs(lead)
        assert n <= 100
        got += raw[pos + 4:pos + 4 + n]
        trail = int(np.frombuffer(raw[pos + 4 + n:pos + 8 + n], ">i4")[0])
        assert abs(trail) == n and (trail < 0) == (k > 0)
        pos += 8 + n
        k += 1
        if lead > 0:
            break
    assert pos == len(raw) and got == payload and k == -(-len(payload) // 100)
    r = evp.read(f, 7, 5, rinv.shape, rinv1.shape, len(ie))
    assert np.array_equal(r["rinv1"], rinv1) and r["oac"] is None


def test_shape_mismatch_and_missing_file(tmp_path):
    planes, rinv, rinv1, ie = _arrays()
    f = tmp_path / "EVP"
    evp.write(f, *planes[:5], rinv, rinv1, ie)
    with pytest.raises(native.SevpError):
        evp.read(f, 7, 5, (4, 7, 7), rinv1.shape, len(ie))
    with pytest.raises(native.SevpError):
        evp.read(tmp_path / "none", 7, 5, rinv.shape, rinv1.shape, len(ie))


def test_pre1_influence_round_trip(tmp_path, oracle):
    """PRE1 influence data of the 96x96 basin (4 blocks) survives the file."""
    p = P.basin(0)
    i2, j2 = p.nx, p.ny
    ie, ok = oracle.block_partition(j2, 4)
    assert ok
    rinv, rinv1, st = oracle.pre1(p.al, p.ab, p.ac, p.ar, p.at, ie)
    assert st == 0
    f = tmp_path / "EVP"
    evp.write(f, p.al, p.ar, p.ab, p.at, p.ac, rinv, rinv1, ie)
    r = evp.read(f, i2, j2, rinv.shape, rinv1.shape, len(ie))
    assert np.array_equal(r["rinv"], rinv) and np.array_equal(r["rinv1"], rinv1)
    assert np.array_equal(r["ac"], p.ac.astype(np.float32)) and np.array_equal(r["ie"], ie)
