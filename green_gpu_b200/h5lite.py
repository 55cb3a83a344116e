"""Minimal read-only HDF5 reader (no libhdf5 / h5py dependency).

Reads the files green-mbpt writes for the density-fitted integrals and its inputs:
superblock v0/v1, version-1 object headers, old-style (symbol-table) groups,
fixed-point / floating-point / compound datatypes, and contiguous, compact or chunked
(unfiltered) layouts.  Used by df_integral.py and by the golden-fixture script.
"""
import numpy as np


class H5File:
    def __init__(self, path):
        with open(path, "rb") as f:
            self.buf = f.read()
        sig = b"\x89HDF\r\n\x1a\n"
        base = None
        for off in (0, 512, 1024, 2048, 4096):
            if self.buf[off:off + 8] == sig:
                base = off
                break
        if base is None:
            raise ValueError(f"{path}: not an HDF5 file")
        p = base + 8
        ver = self.buf[p]
        if ver not in (0, 1):
            raise NotImplementedError(f"superblock version {ver}")
        self.so = self.buf[p + 5]
        self.sl = self.buf[p + 6]
        p += 8 + 4 + 4  # versions/sizes, leaf/internal K, consistency flags
        if ver == 1:
            p += 4
        p += 4 * self.so  # base, free-space, eof, driver addresses
        _, hdr, ctype, scratch = self._symbol_entry(p)
        self.root = hdr

    # -- primitive readers -------------------------------------------------
    def _u(self, p, n):
        return int.from_bytes(self.buf[p:p + n], "little")

    def _symbol_entry(self, p):
        so = self.so
        name_off = self._u(p, so)
        hdr = self._u(p + so, so)
        ctype = self._u(p + 2 * so, 4)
        scratch = self.buf[p + 2 * so + 8:p + 2 * so + 24]
        return name_off, hdr, ctype, scratch

    def _messages(self, addr):
        """Yield (type, data_offset, size) for every message of a v1 object header."""
        ver = self.buf[addr]
        if ver != 1:
            raise NotImplementedError(f"object header version {ver}")
        nmsg = self._u(addr + 2, 2)
        hsize = self._u(addr + 8, 4)
        blocks = [(addr + 16, hsize)]
        seen = 0
        while blocks and seen < nmsg:
            start, length = blocks.pop(0)
            p = start
            while p < start + length and seen < nmsg:
                mtype = self._u(p, 2)
                msize = self._u(p + 2, 2)
                data = p + 8
                seen += 1
                if mtype == 0x10:  # continuation
                    blocks.append((self._u(data, self.so), self._u(data + self.so, self.sl)))
                else:
                    yield mtype, data, msize
                p = data + msize

    def _heap_name(self, heap_addr, off):
        assert self.buf[heap_addr:heap_addr + 4] == b"HEAP"
        data_addr = self._u(heap_addr + 8 + 2 * self.sl, self.so)
        s = data_addr + off
        e = self.buf.index(b"\x00", s)
        return self.buf[s:e].decode()

    def _group_children(self, hdr):
        btree = heap = None
        for mtype, p, _ in self._messages(hdr):
            if mtype == 0x11:
                btree = self._u(p, self.so)
                heap = self._u(p + self.so, self.so)
        if btree is None:
            return None
        out = {}
        self._walk_group_btree(btree, heap, out)
        return out

    def _walk_group_btree(self, node, heap, out):
        assert self.buf[node:node + 4] == b"TREE", "bad group B-tree node"
        level = self.buf[node + 5]
        used = self._u(node + 6, 2)
        p = node + 8 + 2 * self.so
        for _ in range(used):
            p += self.sl  # key
            child = self._u(p, self.so)
            p += self.so
            if level > 0:
                self._walk_group_btree(child, heap, out)
            else:
                assert self.buf[child:child + 4] == b"SNOD"
                nsym = self._u(child + 6, 2)
                q = child + 8
                esize = 2 * self.so + 24
                for _i in range(nsym):
                    name_off, hdr, _, _ = self._symbol_entry(q)
                    out[self._heap_name(heap, name_off)] = hdr
                    q += esize

    # -- datatypes ----------------------------------------------------------
    def _dtype(self, p):
        cls_ver = self.buf[p]
        cls = cls_ver & 0x0F
        ver = cls_ver >> 4
        bits = self._u(p + 1, 3)
        size = self._u(p + 4, 4)
        order = ">" if (bits & 1) else "<"
        if cls == 0:
            signed = (bits >> 3) & 1
            return np.dtype(f"{order}{'i' if signed else 'u'}{size}")
        if cls == 1:
            return np.dtype(f"{order}f{size}")
        if cls == 6:
            nmemb = bits & 0xFFFF
            q = p + 8
            names, fmts, offs = [], [], []
            for _ in range(nmemb):
                e = self.buf.index(b"\x00", q)
                name = self.buf[q:e].decode()
                if ver < 3:
                    q += ((e - q) // 8 + 1) * 8
                else:
                    q = e + 1
                if ver < 3:
                    off = self._u(q, 4)
                    q += 4
                else:
                    nb = max(1, (size.bit_length() + 7) // 8)
                    off = self._u(q, nb)
                    q += nb
                if ver == 1:
                    q += 28
                mdt = self._dtype(q)
                q += 8 + self._dtype_props_len(q)
                names.append(name)
                fmts.append(mdt)
                offs.append(off)
            return np.dtype({"names": names, "formats": fmts, "offsets": offs, "itemsize": size})
        if cls == 3:
            return np.dtype(f"S{size}")
        raise NotImplementedError(f"datatype class {cls}")

    def _dtype_props_len(self, p):
        cls = self.buf[p] & 0x0F
        if cls == 0:
            return 4
        if cls == 1:
            return 12
        if cls == 3:
            return 0
        if cls == 6:
            ver = self.buf[p] >> 4
            bits = self._u(p + 1, 3)
            size = self._u(p + 4, 4)
            q = p + 8
            for _ in range(bits & 0xFFFF):
                e = self.buf.index(b"\x00", q)
                if ver < 3:
                    q += ((e - q) // 8 + 1) * 8 + 4
                else:
                    q = e + 1 + max(1, (size.bit_length() + 7) // 8)
                if ver == 1:
                    q += 28
                q += 8 + self._dtype_props_len(q)
            return q - (p + 8)
        raise NotImplementedError(f"datatype class {cls}")

    # -- datasets -------------------------------------------------------------
    def _read_dataset(self, hdr):
        shape = dtype = None
        layout = None
        for mtype, p, size in self._messages(hdr):
            if mtype == 0x01:
                ver = self.buf[p]
                nd = self.buf[p + 1]
                q = p + (8 if ver == 1 else 4)
                shape = tuple(self._u(q + i * self.sl, self.sl) for i in range(nd))
            elif mtype == 0x03:
                dtype = self._dtype(p)
            elif mtype == 0x08:
                layout = p
            elif mtype == 0x0B:
                raise NotImplementedError("filtered datasets are not supported")
        if shape is None or dtype is None or layout is None:
            return None
        n = int(np.prod(shape)) if shape else 1
        nbytes = n * dtype.itemsize
        ver = self.buf[layout]
        if ver == 3:
            cls = self.buf[layout + 1]
            if cls == 0:
                sz = self._u(layout + 2, 2)
                raw = self.buf[layout + 4:layout + 4 + sz]
            elif cls == 1:
                addr = self._u(layout + 2, self.so)
                raw = self.buf[addr:addr + nbytes] if addr != (1 << (8 * self.so)) - 1 else bytes(nbytes)
            elif cls == 2:
                nd = self.buf[layout + 2]
                addr = self._u(layout + 3, self.so)
                cdims = [self._u(layout + 3 + self.so + 4 * i, 4) for i in range(nd)]
                raw = self._read_chunked(addr, shape, cdims[:-1], dtype)
            else:
                raise NotImplementedError(f"layout class {cls}")
        elif ver in (1, 2):
            nd = self.buf[layout + 1]
            cls = self.buf[layout + 2]
            q = layout + 8
            if cls == 1:
                addr = self._u(q, self.so)
                raw = self.buf[addr:addr + nbytes]
            elif cls == 0:
                q += 4 * nd
                sz = self._u(q, 4)
                raw = self.buf[q + 4:q + 4 + sz]
            else:
                addr = self._u(q, self.so)
                cdims = [self._u(q + self.so + 4 * i, 4) for i in range(nd)]
                raw = self._read_chunked(addr, shape, cdims[:-1], dtype)
        else:
            raise NotImplementedError(f"layout version {ver}")
        return np.frombuffer(raw, dtype=dtype, count=n).reshape(shape).copy()

    def _read_chunked(self, btree, shape, cdims, dtype):
        out = np.zeros(shape, dtype=dtype)
        nd = len(shape)

        def walk(node):
            assert self.buf[node:node + 4] == b"TREE"
            level = self.buf[node + 5]
            used = self._u(node + 6, 2)
            p = node + 8 + 2 * self.so
            ksize = 8 + 8 * (nd + 1)
            for _ in range(used):
                csize = self._u(p, 4)
                offs = [self._u(p + 8 + 8 * i, 8) for i in range(nd)]
                child = self._u(p + ksize, self.so)
                p += ksize + self.so
                if level > 0:
                    walk(child)
                else:
                    chunk = np.frombuffer(self.buf[child:child + csize], dtype=dtype,
                                          count=int(np.prod(cdims))).reshape(cdims)
                    sl = tuple(slice(o, min(o + c, s)) for o, c, s in zip(offs, cdims, shape))
                    sub = tuple(slice(0, s.stop - s.start) for s in sl)
                    out[sl] = chunk[sub]

        walk(btree)
        return out.tobytes()

    # -- public API -------------------------------------------------------------
    def keys(self, path="/"):
        hdr = self._resolve(path)
        ch = self._group_children(hdr)
        return sorted(ch) if ch else []

    def _resolve(self, path):
        hdr = self.root
        for part in [x for x in path.split("/") if x]:
            ch = self._group_children(hdr)
            if ch is None or part not in ch:
                raise KeyError(path)
            hdr = ch[part]
        return hdr

    def __getitem__(self, path):
        hdr = self._resolve(path)
        if self._group_children(hdr) is not None:
            raise KeyError(f"{path} is a group")
        arr = self._read_dataset(hdr)
        if arr is not None and arr.dtype.names and set(arr.dtype.names) >= {"r", "i"}:
            arr = arr["r"].astype(np.float64) + 1j * arr["i"].astype(np.float64)
        return arr

    def walk(self, path="/", prefix=""):
        hdr = self._resolve(path)
        ch = self._group_children(hdr)
        out = []
        for name in sorted(ch):
            full = prefix + "/" + name
            sub = self._group_children(ch[name])
            if sub is not None:
                out += self.walk(full, full)
            else:
                out.append(full)
        return out

