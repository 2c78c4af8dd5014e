"""Result files (rf_write_result_grid; writeResultFile_RF.f90:737-938,
1758-1849), host only.

No HDF5 library exists in this environment, so the HDF5 file is read back by
the small reader below, written from the HDF5 file-format specification
(superblock version 0, version-1 object headers, v1 B-tree, local heap,
symbol-table node, dataspace/datatype/fill/layout/attribute messages): it
checks every signature, version, size and alignment the writer relies on,
finds "samples" through the root group's B-tree and heap, and compares the
data bitwise.  The XDMF file is parsed as XML.
"""
import struct
import xml.etree.ElementTree as ET

import numpy as np
import pytest

import randomfield_b200 as rf

UNDEF = 0xFFFFFFFFFFFFFFFF


class H5:
    def __init__(self, path):
        self.b = open(path, "rb").read()

    def u(self, fmt, at):
        return struct.unpack_from("<" + fmt, self.b, at)

    def superblock(self):
        b = self.b
        assert b[:8] == b"\x89HDF\r\n\x1a\n"
        assert b[8] == 0 and b[9] == 0 and b[10] == 0 and b[12] == 0  # versions
        assert b[13] == 8 and b[14] == 8  # sizes of offsets and lengths
        leafK, internK, flags = self.u("HHI", 16)
        base, freesp, eof, drv = self.u("QQQQ", 24)
        assert (base, freesp, drv) == (0, UNDEF, UNDEF)
        assert eof == len(b)
        name_off, oh, cache, _ = self.u("QQII", 56)
        btree, heap = self.u("QQ", 80)
        assert cache == 1
        return dict(leafK=leafK, internK=internK, root=oh, btree=btree, heap=heap)

    def object_header(self, at):
        assert at % 8 == 0
        ver, _, nmsg, refc, size, pad = struct.unpack_from("<BBHIII", self.b, at)
        assert ver == 1 and refc >= 1 and pad == 0
        msgs, p, end = [], at + 16, at + 16 + size
        for _ in range(nmsg):
            t, sz, fl = struct.unpack_from("<HHB", self.b, p)
            assert sz % 8 == 0 and (p - at) % 8 == 0
            msgs.append((t, fl, self.b[p + 8:p + 8 + sz]))
            p += 8 + sz
        assert p == end
        return msgs

    @staticmethod
    def datatype(d):
        cls, ver = d[0] & 0x0F, d[0] >> 4
        assert ver == 1
        size = struct.unpack_from("<I", d, 4)[0]
        if cls == 1:
            assert d[1:4] == bytes([0x20, 63, 0]) and size == 8
            assert struct.unpack_from("<HHBBBBI", d, 8) == (0, 64, 52, 11, 0, 52, 1023)
            return "<f8"
        assert cls == 0 and d[1] == 0x08 and size == 4 and struct.unpack_from("<HH", d, 8) == (0, 32)
        return "<i4"

    @staticmethod
    def dataspace(d):
        ver, rank, flags = d[0], d[1], d[2]
        assert ver == 1 and flags == 0
        return tuple(struct.unpack_from("<" + "Q" * rank, d, 8))

    @staticmethod
    def attribute(d):
        ver, _, nsz, tsz, ssz = struct.unpack_from("<BBHHH", d, 0)
        assert ver == 1
        p = 8
        name = d[p:p + nsz - 1].decode()
        assert d[p + nsz - 1] == 0
        p += -(-nsz // 8) * 8
        dt = H5.datatype(d[p:p + tsz])
        p += -(-tsz // 8) * 8
        dims = H5.dataspace(d[p:p + ssz])
        p += -(-ssz // 8) * 8
        count = int(np.prod(dims)) if dims else 1
        val = np.frombuffer(d, dtype=dt, count=count, offset=p)
        return name, (val[0] if not dims else val.copy())

    def read(self):
        sb = self.superblock()
        msgs = self.object_header(sb["root"])
        stab = [m for m in msgs if m[0] == 0x0011]
        assert len(stab) == 1
        btree, heap = struct.unpack_from("<QQ", stab[0][2], 0)
        assert (btree, heap) == (sb["btree"], sb["heap"])
        attrs = dict(self.attribute(m[2]) for m in msgs if m[0] == 0x000C)
        # local heap
        assert self.b[heap:heap + 4] == b"HEAP" and self.b[heap + 4] == 0
        dsize, free, daddr = self.u("QQQ", heap + 8)
        assert free == 1  # no free block (the library's end-of-free-list marker)
        seg = self.b[daddr:daddr + dsize]
        assert seg[0] == 0  # the root's empty name

        def name(off):
            assert off % 8 == 0
            return seg[off:seg.index(b"\0", off)].decode()

        # B-tree node: group node, leaf level
        assert self.b[btree:btree + 4] == b"TREE"
        ntype, level, used = struct.unpack_from("<BBH", self.b, btree + 4)
        left, right = self.u("QQ", btree + 8)
        assert (ntype, level, left, right) == (0, 0, UNDEF, UNDEF) and used == 1
        key0, child, key1 = self.u("QQQ", btree + 24)
        assert name(key0) == ""
        # symbol table node
        assert self.b[child:child + 4] == b"SNOD" and self.b[child + 4] == 1
        nsym = self.u("H", child + 6)[0]
        entries = {}
        for i in range(nsym):
            off, oh, cache, _ = self.u("QQII", child + 8 + 40 * i)
            assert cache == 0
            entries[name(off)] = oh
        assert name(key1) == max(entries)
        data = {}
        for nm, oh in entries.items():
            m = {t: body for t, fl, body in self.object_header(oh)}
            dims = self.dataspace(m[0x0001])
            dt = self.datatype(m[0x0003])
            fill = m[0x0005]
            assert fill[0] == 2
            lay = m[0x0008]
            assert lay[0] == 3 and lay[1] == 1
            addr, size = struct.unpack_from("<QQ", lay, 2)
            assert size == 8 * int(np.prod(dims)) and addr + size <= len(self.b)
            data[nm] = np.frombuffer(self.b, dtype=dt, count=int(np.prod(dims)), offset=addr).reshape(dims)
        return data, attrs


def test_h5_and_xmf_3d(tmp_path):
    xMin, xMax, xStep = (0.0, -1.0, 2.0), (0.4, 0.5, 2.6), (0.1, 0.25, 0.2)
    N = [int(round((b - a) / h)) + 1 for a, b, h in zip(xMin, xMax, xStep)]  # 5, 7, 4
    field = np.random.RandomState(3).normal(size=int(np.prod(N)))
    attrs = dict(nb_procs=1, nDim=3, Nmc=4, method=2, seedStart=7, corrMod=1, margiFirst=2, localizationLevel=0,
                 kNStep=(24, 20, 16), nFields=(1, 1, 1), xMinGlob=xMin, xMaxGlob=xMax, xStep=xStep,
                 corrL=(2.0, 1.0, 0.5), overlap=(0.0, 0.0, 0.0), procExtent=(0.4, 1.5, 0.6),
                 kMax_out=(7.355, 7.355, 7.355))
    rf.write_result_grid(str(tmp_path), "field_1", xMin, xMax, xStep, field, attributes=attrs)
    data, got = H5(tmp_path / "h5" / "field_1.h5").read()
    assert list(data) == ["samples"]
    s = data["samples"]
    assert s.shape == (N[2], N[1], N[0])  # slowest axis first
    np.testing.assert_array_equal(s.reshape(-1), field)  # axis 1 fastest, bitwise
    for k in ("nb_procs", "nDim", "Nmc", "method", "seedStart", "corrMod", "margiFirst", "localizationLevel"):
        assert int(got[k]) == attrs[k], k
    for k in ("kNStep", "nFields"):
        np.testing.assert_array_equal(got[k], attrs[k])
    for k in ("xMinGlob", "xMaxGlob", "xStep", "corrL", "overlap", "procExtent", "kMax_out"):
        np.testing.assert_array_equal(got[k], np.asarray(attrs[k], dtype=np.float64))
    # XDMF
    root = ET.parse(tmp_path / "xmf" / "field_1.xmf").getroot()
    assert root.tag == "Xdmf" and root.get("Version") == "2.0"
    item = root.find("Domain/DataItem")
    assert item.get("Name") == "RF_1" and item.get("Format") == "HDF" and item.get("Precision") == "8"
    assert item.get("Dimensions") == f"{N[2]} {N[1]} {N[0]}"
    assert item.text.strip() == "../h5/field_1.h5:/samples"
    grid = root.find("Domain/Grid/Grid")
    topo = grid.find("Topology")
    assert topo.get("TopologyType") == "3DCoRectMesh" and topo.get("Dimensions") == f"{N[2]} {N[1]} {N[0]}"
    geo = grid.find("Geometry")
    assert geo.get("GeometryType") == "ORIGIN_DXDYDZ"
    origin, step = geo.findall("DataItem")
    np.testing.assert_array_equal([float(v) for v in origin.text.split()], xMin[::-1])
    np.testing.assert_array_equal([float(v) for v in step.text.split()], xStep[::-1])
    att = grid.find("Attribute")
    assert att.get("Name") == "RF1" and att.get("Center") == "Node"
    assert att.find("DataItem").text.strip() == '/Xdmf/Domain/DataItem[@Name="RF_1"]'


def test_h5_2d_without_attributes_and_1d_without_xmf(tmp_path):
    field = np.arange(6 * 3, dtype=np.float64) * 0.5 - 2.0
    rf.write_result_grid(str(tmp_path), "f2", (0.0, 0.0), (0.5, 0.2), (0.1, 0.1), field)
    data, attrs = H5(tmp_path / "h5" / "f2.h5").read()
    assert attrs == {}
    np.testing.assert_array_equal(data["samples"], field.reshape(3, 6))
    root = ET.parse(tmp_path / "xmf" / "f2.xmf").getroot()
    assert root.find("Domain/Grid/Grid/Topology").get("TopologyType") == "2DCoRectMesh"
    f1 = np.linspace(-1, 1, 11)
    (tmp_path / "one").mkdir()
    rf.write_result_grid(str(tmp_path / "one"), "f1", (0.0,), (1.0,), (0.1,), f1)
    data, _ = H5(tmp_path / "one" / "h5" / "f1.h5").read()
    np.testing.assert_array_equal(data["samples"], f1)
    assert not (tmp_path / "one" / "xmf").exists()  # no XDMF model for 1-D in the reference


def test_writer_errors(tmp_path):
    with pytest.raises(rf.RandomFieldError) as e:
        rf.write_result_grid(str(tmp_path / "missing" / "deeper"), "x", (0.0, 0.0), (1.0, 1.0), (0.5, 0.5),
                             np.zeros(9))
    assert e.value.code == -9
    with pytest.raises(rf.RandomFieldError) as e:
        rf.write_result_grid(str(tmp_path), "x", (0.0, 0.0), (1.0, 1.0), (0.5, 0.5), np.zeros(8))
    assert e.value.code == -9
    with pytest.raises(rf.RandomFieldError) as e:
        rf.write_result_grid(str(tmp_path), "x", (0.0, 0.0), (1.0, 1.0), (0.0, 0.5), np.zeros(9))
    assert e.value.code == -9
