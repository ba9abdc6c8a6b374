"""Reader and writer of the bsr_mat.nnn interaction-matrix file.

bsr_mat writes one file per partial wave and bsr_hd reads it (the only
interface between the two programs of the hot path):

  write(nui) ns, nch, kcp                        sub1.f90:110-112
  Record_matrix (overlap)                        record_matrix.f90:2-59
  Record_matrix (interaction)                    sub1.f90:202
  write(nui) mk; write(nui) ACF; write(nui) t(ns+1), ns      sub1.f90:262
  write(nui) htarg; write(nui) otarg; write(nui) Etarg; write(nui) EC   sub1.f90:268-272

Record_matrix writes the nch diagonal blocks hcc(:,:,i(i+1)/2) (one record
each), then for every non-zero off-diagonal block (ich > jch) a record
(ich, jch) followed by the block, and ends with the record (0, idiag), idiag = 1
when no off-diagonal block was written.  bsr_hd reads the same sequence
(diag_hd.f90:36-64) and takes the trailing idiag of the overlap as diag_ovl.

The records use gfortran's unformatted sequential layout: a 4-byte length, the
payload, the same 4-byte length (little-endian; default Integer is 4 bytes,
Real(8) 8 bytes).  Perturbers (kcp > 0) are outside the benchmark workloads and
are rejected.
"""
import struct

import numpy as np


def _rec(f, payload):
    f.write(struct.pack("<i", len(payload)))
    f.write(payload)
    f.write(struct.pack("<i", len(payload)))


def _read_rec(f):
    h = f.read(4)
    if len(h) < 4:
        raise EOFError("bsr_mat: unexpected end of file")
    n = struct.unpack("<i", h)[0]
    if n < 0:
        raise ValueError("bsr_mat: record split into sub-records is not supported")
    data = f.read(n)
    t = f.read(4)
    if len(data) != n or len(t) != 4 or struct.unpack("<i", t)[0] != n:
        raise ValueError("bsr_mat: corrupt record markers")
    return data


def _blocks(blk, nch):
    """blk: (nblk, ns, ns) [row, col] in hcc block order -> (diag list, {(i,j): block})."""
    diag = [blk[i * (i + 1) // 2 + i] for i in range(nch)]
    off = {}
    for i in range(1, nch):
        for j in range(i):
            off[(i + 1, j + 1)] = blk[i * (i + 1) // 2 + j]
    return diag, off


def _record_matrix(f, blk, nch):
    diag, off = _blocks(blk, nch)
    for d in diag:
        _rec(f, np.asfortranarray(d, dtype="<f8").tobytes(order="F"))
    idiag = 1
    for (i, j), b in off.items():
        if np.sum(np.abs(b)) == 0.0:
            continue
        _rec(f, struct.pack("<2i", i, j))
        _rec(f, np.asfortranarray(b, dtype="<f8").tobytes(order="F"))
        idiag = 0
    _rec(f, struct.pack("<2i", 0, idiag))


def write_bsr_mat(path, scc, hcc, nch, ns, acf, rmax, htarg=None, otarg=None, etarg=None, ec=0.0):
    """Write bsr_mat.nnn.  scc, hcc: (nch(nch+1)/2, ns, ns) blocks [row, col];
    acf: (nch, nch, mk+1); rmax = t(ns+1)."""
    nblk = nch * (nch + 1) // 2
    scc = np.asarray(scc, dtype=np.float64).reshape(nblk, ns, ns)
    hcc = np.asarray(hcc, dtype=np.float64).reshape(nblk, ns, ns)
    acf = np.asarray(acf, dtype=np.float64)
    mk = acf.shape[2] - 1
    htarg = np.zeros(nblk) if htarg is None else np.asarray(htarg, dtype=np.float64)
    otarg = np.zeros(nblk) if otarg is None else np.asarray(otarg, dtype=np.float64)
    etarg = np.zeros(1) if etarg is None else np.asarray(etarg, dtype=np.float64)
    with open(path, "wb") as f:
        _rec(f, struct.pack("<3i", ns, nch, 0))
        _record_matrix(f, scc, nch)
        _record_matrix(f, hcc, nch)
        _rec(f, struct.pack("<i", mk))
        _rec(f, np.asfortranarray(acf, dtype="<f8").tobytes(order="F"))
        _rec(f, struct.pack("<di", float(rmax), ns))
        _rec(f, htarg.astype("<f8").tobytes())
        _rec(f, otarg.astype("<f8").tobytes())
        _rec(f, etarg.astype("<f8").tobytes())
        _rec(f, struct.pack("<d", float(ec)))


def _read_matrix(f, ns, nch):
    nblk = nch * (nch + 1) // 2
    blk = np.zeros((nblk, ns, ns))
    for i in range(nch):
        d = np.frombuffer(_read_rec(f), dtype="<f8")
        blk[i * (i + 1) // 2 + i] = d.reshape((ns, ns), order="F")
    while True:
        ic, jc = struct.unpack("<2i", _read_rec(f))
        if ic <= 0:
            return blk, jc
        if ic > nch or jc > nch or jc >= ic:
            raise ValueError("bsr_mat: block (%d,%d) outside the channel blocks" % (ic, jc))
        b = np.frombuffer(_read_rec(f), dtype="<f8").reshape((ns, ns), order="F")
        blk[(ic - 1) * ic // 2 + jc - 1] = b


def read_bsr_mat(path):
    """Read bsr_mat.nnn as written by bsr_mat (or write_bsr_mat)."""
    with open(path, "rb") as f:
        ns, nch, kcp = struct.unpack("<3i", _read_rec(f))
        if kcp != 0:
            raise NotImplementedError("bsr_mat: perturbers (kcp=%d) are not supported" % kcp)
        scc, diag_ovl = _read_matrix(f, ns, nch)
        hcc, diag_hm = _read_matrix(f, ns, nch)
        (mk,) = struct.unpack("<i", _read_rec(f))
        acf = np.frombuffer(_read_rec(f), dtype="<f8").reshape((nch, nch, mk + 1), order="F").copy()
        rmax, ns2 = struct.unpack("<di", _read_rec(f))
        htarg = np.frombuffer(_read_rec(f), dtype="<f8").copy()
        otarg = np.frombuffer(_read_rec(f), dtype="<f8").copy()
        etarg = np.frombuffer(_read_rec(f), dtype="<f8").copy()
        (ec,) = struct.unpack("<d", _read_rec(f))
    return {"ns": ns, "nch": nch, "kcp": kcp, "scc": scc, "hcc": hcc, "diag_ovl": diag_ovl, "diag_hm": diag_hm,
            "mk": mk, "acf": acf, "rmax": rmax, "htarg": htarg, "otarg": otarg, "etarg": etarg, "ec": ec}
