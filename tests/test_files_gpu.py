"""TNL's binary matrix file (SparseMatrix::save / load) against the
reference's own Host save of the same matrix (oracle/_ref):

* save: the file's bytes equal the reference's -- except bytes the
  reference never initialises (ChunkedEllpack slice records past
  numberOfSlices, AdaptiveCSR descriptor fields a descriptor type leaves
  unset, and padding), which are compared where defined;
* load of the reference's file: the same metadata, values and columns as the
  matrix built here, the same product, and a save of it gives the same bytes;
* a file of another matrix type is refused with the reference's message.
"""
import struct

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

FMTS = {"CSR": 0, "Ellpack": 1, "SlicedEllpack": 2, "ChunkedEllpack": 3, "BiEllpack": 4, "AdaptiveCSR": 5}


def tnl():
    import tnl_b200

    return tnl_b200


def parse(b: bytes):
    """Objects of a TNL file: (type string, payload bytes) plus raw scalar runs."""
    out, i = [], 0
    while i < len(b):
        if b[i:i + 5] == b"TNLMN":
            n = struct.unpack_from("<i", b, i + 5)[0]
            t = b[i + 9:i + 9 + n].decode()
            i += 9 + n
            if t.startswith("TNL::Containers::Array"):
                cnt = struct.unpack_from("<Q", b, i)[0]
                i += 8
                el = 20 if "Descriptor" in t else 16 if "SliceInfo" in t else 8 if "double" in t else 4
                out.append((t, b[i:i + cnt * el]))
                i += cnt * el
            else:
                out.append((t, b""))
        else:
            j = b.find(b"TNLMN", i)
            j = len(b) if j < 0 else j
            out.append(("raw", b[i:j]))
            i = j
    return out


def masked(objs, nslices=None):
    """Zero the bytes the reference leaves unset."""
    res = []
    for t, p in objs:
        if "SliceInfo" in t and nslices is not None:
            p = p[:16 * nslices] + bytes(len(p) - 16 * nslices)
        if "Descriptor" in t:
            q = bytearray(p)
            for k in range(len(q) // 20):
                d = q[20 * k:20 * k + 20]
                typ = d[0]
                keep = bytearray(20)
                keep[0] = d[0]
                keep[4:8] = d[4:8]  # first segment
                keep[16] = d[16]  # warp index
                last = k == len(q) // 20 - 1
                if typ != 0 and not last:
                    keep[8:16] = d[8:16]  # block size, segments in block
                if typ == 0:
                    keep[17] = d[17]  # warps count
                q[20 * k:20 * k + 20] = keep
            p = bytes(q)
        res.append((t, p))
    return res


def matrices():
    from tnl_b200 import generators as g

    return {"laplacian20": g.laplacian_2d(20), "powerlaw": g.power_law(3000, 1.73, 200, 9)}


@pytest.mark.parametrize("fmt", list(FMTS))
@pytest.mark.parametrize("org", ["col", "row"])
@pytest.mark.parametrize("real", [np.float64, np.float32])
def test_save_matches_reference_and_load_round_trips(reference, tmp_path, fmt, org, real):
    t = tnl()
    if org == "row" and fmt in ("CSR", "AdaptiveCSR"):
        pytest.skip("the CSR formats have no organization")
    tdt = torch.float64 if real == np.float64 else torch.float32
    ORG = t.RowMajorOrder if org == "row" else t.ColumnMajorOrder
    for name, A in matrices().items():
        vals = A.vals.astype(real)
        M = t.SparseMatrix(t.FORMATS[fmt], tdt, ORG).assign(A.rowptr, A.cols, vals, A.ncols)
        mine, ref = tmp_path / f"{name}.mine.tnl", tmp_path / f"{name}.ref.tnl"
        M.save(mine)
        reference.save(FMTS[fmt], A, ref, colmajor=(org == "col"), real64=(real == np.float64))
        bm, br = mine.read_bytes(), ref.read_bytes()
        nsl = M.segments.info.slices if fmt == "ChunkedEllpack" else None
        if fmt in ("ChunkedEllpack", "AdaptiveCSR"):
            assert masked(parse(bm), nsl) == masked(parse(br), nsl), (name, fmt)
        else:
            assert bm == br, (name, fmt)
        # load the reference's file into a matrix of the same type
        L = t.SparseMatrix(t.FORMATS[fmt], tdt, ORG).load(ref)
        assert L.getRows() == A.n and L.getColumns() == A.ncols
        assert torch.equal(L.getValues(), M.getValues()) and torch.equal(L.getColumnIndexes(), M.getColumnIndexes())
        x = torch.tensor(np.random.default_rng(1).uniform(-1, 1, A.ncols).astype(real), device="cuda")
        y1 = torch.zeros(A.n, dtype=tdt, device="cuda")
        y2 = torch.zeros(A.n, dtype=tdt, device="cuda")
        M.vectorProduct(x, y1)
        L.vectorProduct(x, y2)
        assert torch.equal(y1, y2), (name, fmt)
        again = tmp_path / f"{name}.again.tnl"
        L.save(again)
        assert again.read_bytes() == bm, (name, fmt)


def test_load_refuses_another_type(reference, tmp_path):
    t = tnl()
    from tnl_b200 import generators as g

    A = g.laplacian_2d(10)
    path = tmp_path / "csr.tnl"
    reference.save(0, A, path)
    with pytest.raises(RuntimeError, match="object type does not match"):
        t.SparseMatrix(t.Ellpack, torch.float64).load(path)
    with pytest.raises(RuntimeError, match="object type does not match"):
        t.SparseMatrix(t.CSR, torch.float32).load(path)
    L = t.SparseMatrix(t.CSR, torch.float64).load(path)
    assert L.getRows() == A.n


@pytest.mark.parametrize("bad_column", [-2, 100])
def test_load_rejects_column_indexes_outside_the_matrix(tmp_path, bad_column):
    """A file whose column array holds an index below the padding value -1
    or at least the column count is reported as corrupt before anything is
    copied to the device: the products gather x[column] unchecked."""
    t = tnl()
    from tnl_b200 import generators as g

    A = g.laplacian_2d(10)
    M = t.SparseMatrix(t.CSR, torch.float64).assign(A.rowptr, A.cols, A.vals, A.ncols)
    good = tmp_path / "good.tnl"
    M.save(good)
    raw = good.read_bytes()
    cols = np.ascontiguousarray(A.cols, np.int32).tobytes()
    at = raw.find(cols)
    assert at > 0 and raw.find(cols, at + 1) < 0
    patched = raw[:at] + np.int32(bad_column).tobytes() + raw[at + 4:]
    bad = tmp_path / "bad.tnl"
    bad.write_bytes(patched)
    with pytest.raises(RuntimeError, match="not a valid TNL sparse matrix file"):
        t.SparseMatrix(t.CSR, torch.float64).load(bad)
    assert t.SparseMatrix(t.CSR, torch.float64).load(good).getRows() == A.n
