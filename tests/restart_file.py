"""Reader and writer of the WAVES section of a CP-PAW restart file, for tests.

Sequential unformatted Fortran records, each framed by its byte length as a
4-byte integer.  The section is the one WAVES$WRITE (src/paw_waves2.f90:
3058-3088) writes for one k-point, one spin and NDIM = 1: the separator
(src/paw_report.f90:108-115), the records of WAVES_WRITEPSI (:3216-3326) and
of WAVES_WRITELAMBDA (:3974-4025).
"""
import struct

import numpy as np


def read_records(path):
    out = []
    with open(path, "rb") as f:
        data = f.read()
    off = 0
    while off < len(data):
        (n,) = struct.unpack_from("<i", data, off)
        body = data[off + 4:off + 4 + n]
        (m,) = struct.unpack_from("<i", data, off + 4 + n)
        assert m == n, "record markers differ"
        out.append(body)
        off += 8 + n
    return out


def write_records(path, recs):
    with open(path, "wb") as f:
        for r in recs:
            f.write(struct.pack("<i", len(r)) + r + struct.pack("<i", len(r)))


def parse_waves(recs):
    """The section as a dict of numpy arrays; checks every record's length."""
    sep = recs[0]
    assert len(sep) == 4 + 32 + 32 + 64 + 256
    d = {"nrec": struct.unpack_from("<i", sep)[0],
         "id": sep[4:36].decode().rstrip(), "name": sep[36:68].decode().rstrip(),
         "version": sep[68:132].decode().rstrip(), "notes": sep[132:388].decode().rstrip()}
    assert d["nrec"] == len(recs) - 1
    r1 = recs[1]
    assert len(r1) == 84
    d["nkpt"], d["nspin"] = struct.unpack_from("<2i", r1)
    d["rbas"] = np.frombuffer(r1[8:80], dtype="<f8").reshape(3, 3, order="F")
    (d["nwave"],) = struct.unpack_from("<i", r1, 80)
    r2 = recs[2]
    assert len(r2) == 24 and r2[:8] == b"PSI     "
    d["ngg"], d["ndim"], d["nb"], d["tsuper"] = struct.unpack_from("<4i", r2, 8)
    nbh = (d["nb"] + 1) // 2 if d["tsuper"] else d["nb"]
    r3 = recs[3]
    assert len(r3) == 24 + 12 * d["ngg"]
    d["xk"] = np.frombuffer(r3[:24], dtype="<f8")
    d["igvec"] = np.frombuffer(r3[24:], dtype="<i4").reshape(d["ngg"], 3)
    k = 4
    psi = []
    for _ in range(d["nwave"]):
        w = []
        for _ in range(nbh):
            assert len(recs[k]) == 16 * d["ngg"]
            w.append(np.frombuffer(recs[k], dtype="<c16"))
            k += 1
        psi.append(np.array(w))
    d["psi"] = psi
    rl = recs[k]
    assert len(rl) == 24 and rl[:8] == b"LAMBDA  "
    nbl, ndim, nspin, d["nlambda"] = struct.unpack_from("<4i", rl, 8)
    assert nbl == d["nb"] and ndim == 1 and nspin == 1
    k += 1
    lam = []
    for _ in range(d["nlambda"]):
        assert len(recs[k]) == 16 * d["nb"] ** 2
        lam.append(np.frombuffer(recs[k], dtype="<c16").reshape(d["nb"], d["nb"]))
        k += 1
    d["lambda"] = lam
    assert k == len(recs)
    return d


def permuted(recs, perm, keep):
    """The section rewritten with its G vectors in the order `perm` and only the
    first `keep` of them: a file written for another G set of the same cell."""
    d = parse_waves(recs)
    sel = np.asarray(perm)[:keep]
    out = list(recs)
    out[0] = recs[0]
    out[2] = recs[2][:8] + struct.pack("<i", keep) + recs[2][12:]
    out[3] = recs[3][:24] + np.ascontiguousarray(d["igvec"][sel], dtype="<i4").tobytes()
    k = 4
    for w in d["psi"]:
        for band in w:
            out[k] = np.ascontiguousarray(band[sel]).tobytes()
            k += 1
    return out


def static(recs):
    """The section as a static restart writes it (NWAVE = 1: PSI0 only, no PSIM
    records), with NREC of the separator adjusted."""
    d = parse_waves(recs)
    nbh = len(d["psi"][0])
    out = [recs[0], recs[1][:80] + struct.pack("<i", 1)] + list(recs[2:4 + nbh]) + list(recs[4 + 2 * nbh:])
    out[0] = struct.pack("<i", len(out) - 1) + recs[0][4:]
    return out


def damaged(path):
    """(name, bytes) of two corrupt copies of a restart section: NGG = -5 in the
    PSI header, and a G-vector record whose leading length marker claims
    2**31 - 1 bytes."""
    recs = read_records(path)
    neg = list(recs)
    neg[2] = recs[2][:8] + struct.pack("<i", -5) + recs[2][12:]
    raw_neg = b"".join(struct.pack("<i", len(r)) + r + struct.pack("<i", len(r)) for r in neg)
    raw = bytearray(open(path, "rb").read())
    off = sum(8 + len(r) for r in recs[:3])
    struct.pack_into("<i", raw, off, 2**31 - 1)
    return [("neg_ngg.rst", raw_neg), ("huge_rec.rst", bytes(raw))]
