"""Burst ingest from Sentinel-1 measurement TIFFs.

Replaces the reference's ``_stream_tiff_from_zip`` (s1proc/sentinel_scene.py:
164-207) and the ``geo2rdr --stdin`` pipe it feeds (sentinel_scene.py:419-437,
csrc/src/geo2rdr.cu:545-557).  The reference reads each burst through GDAL's
``/vsizip/``, which widens the TIFF's complex int16 samples to complex64 on the
host, and writes 8 bytes per sample into the pipe; the executable copies them
to the GPU burst by burst.  Here:

* ``MeasurementTiff`` parses the TIFF directory itself (classic TIFF or
  BigTIFF, either byte order; uncompressed complex int16 in strips or tiles)
  and reads row ranges straight into caller buffers -- from a plain file, or
  from a member of the SAFE zip (stored members in place, deflated ones
  through zipfile's seekable stream);
* ``BurstStream`` keeps the samples as int16 pairs (4 bytes per sample, half
  the bytes of the pipe) in two pinned host buffers: burst k + 1 is read on a
  reader thread while burst k is copied to the device on a copy stream and
  processed; the widening happens in the deramp (``s1b_deramp_ci16``).
"""
from __future__ import annotations

import os
import struct
import threading
import zipfile
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import torch

# TIFF tags (TIFF 6.0 specification; BigTIFF as published by Aware Systems)
_WIDTH, _LENGTH, _BPS, _COMPRESSION, _SPP, _PLANAR = 256, 257, 258, 259, 277, 284
_STRIP_OFFSETS, _ROWS_PER_STRIP, _STRIP_BYTES = 273, 278, 279
_TILE_WIDTH, _TILE_LENGTH, _TILE_OFFSETS, _TILE_BYTES = 322, 323, 324, 325
_SAMPLE_FORMAT = 339
# field types: code -> (struct letter, size)
_TYPES = {1: ("B", 1), 2: ("c", 1), 3: ("H", 2), 4: ("I", 4), 6: ("b", 1), 7: ("B", 1), 8: ("h", 2),
          9: ("i", 4), 11: ("f", 4), 12: ("d", 8), 16: ("Q", 8), 17: ("q", 8), 18: ("Q", 8)}


class _FileSource:
    """Positional reads of a plain file (os.pread: no shared file position)."""

    def __init__(self, path):
        self.fd = os.open(path, os.O_RDONLY)
        self.size = os.fstat(self.fd).st_size

    def read(self, offset, n):
        b = os.pread(self.fd, n, offset)
        if len(b) != n:
            raise EOFError(f"short read: {len(b)} of {n} bytes at {offset}")
        return b

    def readinto(self, offset, mv):
        got = os.preadv(self.fd, [mv], offset)
        if got != len(mv):
            raise EOFError(f"short read: {got} of {len(mv)} bytes at {offset}")

    def close(self):
        os.close(self.fd)


class _ZipSource:
    """A member of a zip archive.  Stored (uncompressed) members are read in
    place at their data offset; compressed ones through zipfile's seekable
    member stream (forward reads are cheap, backward ones restart the inflate)."""

    def __init__(self, path, member):
        self.zf = zipfile.ZipFile(path)
        info = self.zf.getinfo(member)
        self.size = info.file_size
        self.lock = threading.Lock()
        if info.compress_type == zipfile.ZIP_STORED:
            raw = _FileSource(path)
            hdr = raw.read(info.header_offset, 30)
            if hdr[:4] != b"PK\x03\x04":
                raise ValueError(f"{path}: bad local header for {member}")
            nlen, xlen = struct.unpack("<HH", hdr[26:30])
            self.base = info.header_offset + 30 + nlen + xlen
            self.raw, self.stream = raw, None
        else:
            self.raw, self.stream = None, self.zf.open(member)

    def read(self, offset, n):
        if self.raw is not None:
            return self.raw.read(self.base + offset, n)
        with self.lock:
            self.stream.seek(offset)
            b = self.stream.read(n)
        if len(b) != n:
            raise EOFError(f"short read: {len(b)} of {n} bytes at {offset}")
        return b

    def readinto(self, offset, mv):
        if self.raw is not None:
            self.raw.readinto(self.base + offset, mv)
        else:
            mv[:] = self.read(offset, len(mv))

    def close(self):
        if self.raw is not None:
            self.raw.close()
        if self.stream is not None:
            self.stream.close()
        self.zf.close()


class MeasurementTiff:
    """One band of complex int16 samples in an uncompressed TIFF.

    ``path`` is a TIFF file, or a zip (a SAFE product) with ``member`` the
    measurement TIFF inside it (the reference's ``/vsizip/`` path,
    sentinel_scene.py:177).  Accepts the layouts writers use for CInt16:
    BitsPerSample 32 with SampleFormat 5 (complex integer), or two int16
    samples per pixel (BitsPerSample 16, SamplesPerPixel 2, SampleFormat 2).
    ``width``/``height`` are the raster size in samples and lines.
    """

    def __init__(self, path, member=None):
        self.src = _ZipSource(path, member) if member is not None else _FileSource(path)
        try:
            self._parse()
        except Exception:
            self.src.close()
            raise

    def close(self):
        self.src.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _parse(self):
        head = self.src.read(0, 16)
        bo = {b"II": "<", b"MM": ">"}.get(head[:2])
        if bo is None:
            raise ValueError("not a TIFF (byte-order mark)")
        magic = struct.unpack(bo + "H", head[2:4])[0]
        if magic == 42:
            big, ifd = False, struct.unpack(bo + "I", head[4:8])[0]
        elif magic == 43:
            if struct.unpack(bo + "HH", head[4:8]) != (8, 0):
                raise ValueError("BigTIFF with an offset size other than 8")
            big, ifd = True, struct.unpack(bo + "Q", head[8:16])[0]
        else:
            raise ValueError(f"not a TIFF (magic {magic})")
        self.byteorder = bo
        if big:
            n = struct.unpack(bo + "Q", self.src.read(ifd, 8))[0]
            ent, esize, first, inline = self.src.read(ifd + 8, 20 * n), 20, "HHQ", 8
        else:
            n = struct.unpack(bo + "H", self.src.read(ifd, 2))[0]
            ent, esize, first, inline = self.src.read(ifd + 2, 12 * n), 12, "HHI", 4
        tags = {}
        for k in range(n):
            e = ent[k * esize:(k + 1) * esize]
            tag, typ, count = struct.unpack(bo + first, e[:esize - inline])
            if typ not in _TYPES:
                continue
            letter, size = _TYPES[typ]
            nbytes = size * count
            data = e[esize - inline:esize - inline + nbytes] if nbytes <= inline else \
                self.src.read(struct.unpack(bo + ("Q" if big else "I"), e[esize - inline:])[0], nbytes)
            tags[tag] = struct.unpack(bo + letter * count, data) if letter != "c" else data
        get = lambda t, d=None: tags[t] if t in tags else d  # noqa: E731
        self.width, self.height = int(get(_WIDTH)[0]), int(get(_LENGTH)[0])
        bps = get(_BPS, (1,))
        spp = int(get(_SPP, (1,))[0])
        fmt = get(_SAMPLE_FORMAT, (1,))
        if int(get(_COMPRESSION, (1,))[0]) != 1:
            raise ValueError("compressed TIFF data (only uncompressed measurement TIFFs are read)")
        cint16 = (spp == 1 and int(bps[0]) == 32 and int(fmt[0]) == 5) or \
                 (spp == 2 and all(int(b) == 16 for b in bps) and all(int(f) == 2 for f in fmt) and
                  int(get(_PLANAR, (1,))[0]) == 1)
        if not cint16:
            raise ValueError(f"not complex int16 samples (BitsPerSample {bps}, SamplesPerPixel {spp}, "
                             f"SampleFormat {fmt})")
        if _TILE_OFFSETS in tags:
            self.tiled = True
            self.tile_w, self.tile_h = int(get(_TILE_WIDTH)[0]), int(get(_TILE_LENGTH)[0])
            self.offsets = np.asarray(get(_TILE_OFFSETS), dtype=np.int64)
            self.counts = np.asarray(get(_TILE_BYTES), dtype=np.int64)
            self.tiles_x = (self.width + self.tile_w - 1) // self.tile_w
            need = self.tiles_x * ((self.height + self.tile_h - 1) // self.tile_h)
            if self.offsets.size != need or (self.counts != self.tile_w * self.tile_h * 4).any():
                raise ValueError("tile table does not match the raster")
        else:
            self.tiled = False
            self.rows_per_strip = min(int(get(_ROWS_PER_STRIP, (self.height,))[0]), self.height)
            self.offsets = np.asarray(get(_STRIP_OFFSETS), dtype=np.int64)
            self.counts = np.asarray(get(_STRIP_BYTES), dtype=np.int64)
            nstrip = (self.height + self.rows_per_strip - 1) // self.rows_per_strip
            if self.offsets.size != nstrip or self.counts.size != nstrip:
                raise ValueError("strip table does not match the raster")
            for s in range(nstrip):
                rows = min(self.rows_per_strip, self.height - s * self.rows_per_strip)
                if self.counts[s] < rows * self.width * 4:
                    raise ValueError(f"strip {s} shorter than its rows")

    def read_rows(self, row0, nrows, out=None):
        """Lines [row0, row0 + nrows) as int16 [nrows, width, 2] (re, im),
        into ``out`` (a C-contiguous int16 array or a CPU tensor, e.g. pinned)
        when given."""
        if row0 < 0 or nrows < 0 or row0 + nrows > self.height:
            raise ValueError(f"rows [{row0}, {row0 + nrows}) outside the raster of {self.height} lines")
        if out is None:
            out = np.empty((nrows, self.width, 2), dtype=np.int16)
        arr = out.numpy() if isinstance(out, torch.Tensor) else out
        if arr.dtype != np.int16 or arr.shape != (nrows, self.width, 2) or not arr.flags.c_contiguous:
            raise ValueError("out must be C-contiguous int16 [nrows, width, 2]")
        flat = arr.reshape(nrows, self.width * 2)
        rowbytes = self.width * 4
        if not self.tiled:
            r = row0
            while r < row0 + nrows:
                s = r // self.rows_per_strip
                s_end = min((s + 1) * self.rows_per_strip, self.height, row0 + nrows)
                k = s_end - r
                off = int(self.offsets[s]) + (r - s * self.rows_per_strip) * rowbytes
                self.src.readinto(off, memoryview(flat[r - row0:r - row0 + k]).cast("B"))
                r = s_end
        else:
            tw, th = self.tile_w, self.tile_h
            tile = np.empty((th, tw * 2), dtype=np.int16)
            for ty in range(row0 // th, (row0 + nrows - 1) // th + 1 if nrows else row0 // th):
                r0, r1 = max(row0, ty * th), min(row0 + nrows, (ty + 1) * th)
                for tx in range(self.tiles_x):
                    self.src.readinto(int(self.offsets[ty * self.tiles_x + tx]), memoryview(tile).cast("B"))
                    c1 = min(tw, self.width - tx * tw)
                    flat[r0 - row0:r1 - row0, 2 * tx * tw:2 * (tx * tw + c1)] = \
                        tile[r0 - ty * th:r1 - ty * th, :2 * c1]
        if self.byteorder == ">":
            flat.byteswap(inplace=True)
        return out

    def read_burst(self, index, lines_per_burst, out=None):
        """Burst ``index`` of a TIFF whose bursts are stacked down the lines
        (sentinel_scene.py:182-196: burst k is lines k * L .. (k + 1) * L)."""
        return self.read_rows(index * lines_per_burst, lines_per_burst, out)


class BurstStream:
    """Bursts of a measurement TIFF as device tensors, read ahead.

    Iterating yields (index, int16 [lines_per_burst, width, 2] CUDA tensor)
    for bursts ``indices`` (default: all ``nbursts``) in order.  The yielded
    tensor is valid on the current stream until the next iteration step (two
    device buffers alternate).  Burst k + 1 is read into the other pinned host
    buffer by a reader thread while burst k's copy and processing run; the
    host-to-device copy runs on its own stream, ordered against the current
    stream with events.  ``bytes_read`` counts the sample bytes moved.
    """

    def __init__(self, tiff: MeasurementTiff, lines_per_burst, nbursts, indices=None, device="cuda"):
        if tiff.height < lines_per_burst * nbursts:
            raise ValueError(f"TIFF has {tiff.height} lines, fewer than {nbursts} bursts of {lines_per_burst}")
        self.tiff, self.L, self.n = tiff, int(lines_per_burst), int(nbursts)
        self.indices = list(range(self.n)) if indices is None else [int(i) for i in indices]
        if any(i < 0 or i >= self.n for i in self.indices):
            raise ValueError("burst index out of range")
        self.device = torch.device(device)
        shape = (self.L, tiff.width, 2)
        self.host = [torch.empty(shape, dtype=torch.int16, pin_memory=True) for _ in range(2)]
        self.dev = [torch.empty(shape, dtype=torch.int16, device=self.device) for _ in range(2)]
        self.bytes_read = 0

    def __iter__(self):
        copy = torch.cuda.Stream(self.device)
        h2d = [torch.cuda.Event() for _ in range(2)]
        used = [torch.cuda.Event() for _ in range(2)]
        pending = [False, False]

        def read(slot, index):
            if pending[slot]:
                h2d[slot].synchronize()  # the copy out of this host buffer is done
            self.tiff.read_burst(index, self.L, self.host[slot])

        with ThreadPoolExecutor(max_workers=1) as pool:
            fut = pool.submit(read, 0, self.indices[0]) if self.indices else None
            for k, index in enumerate(self.indices):
                slot = k & 1
                fut.result()
                cur = torch.cuda.current_stream(self.device)
                if k >= 2:
                    copy.wait_event(used[slot])  # burst k - 2's work on this device buffer is done
                with torch.cuda.stream(copy):
                    self.dev[slot].copy_(self.host[slot], non_blocking=True)
                    h2d[slot].record(copy)
                pending[slot] = True
                cur.wait_event(h2d[slot])
                if k + 1 < len(self.indices):
                    fut = pool.submit(read, slot ^ 1, self.indices[k + 1])
                self.bytes_read += self.host[slot].numel() * 2
                yield index, self.dev[slot]
                used[slot].record(torch.cuda.current_stream(self.device))
            torch.cuda.current_stream(self.device).synchronize()
