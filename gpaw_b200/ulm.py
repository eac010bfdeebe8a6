"""The ULM container of GPAW's .gpw files.

GPAW writes its restart files through ase.io.ulm (gpaw/io/__init__.py:1-15,
Calculator.write, gpaw/calculator.py:294-325); ASE is not a dependency of
this package, so the container is read and written here from its published
layout (ULM file format version 3, ASE >= 3.15):

  bytes 0-7     b'- of Ulm'
  bytes 8-23    tag, ASCII, space padded ('GPAW' for GPAW's files)
  bytes 24-47   three little-endian int64: format version (3), number of
                items, file offset of the item table
  arrays        raw C-order data, each starting at an 8-byte aligned offset
  items         per item: an int64 byte count and a UTF-8 JSON object; a key
                ending in '.' holds either a nested object (a child) or
                {"ndarray": [shape, dtype name, offset]} (an array in the
                file); plain keys hold JSON values (complex numbers as
                {"__complex__": [re, im]}, small arrays inline as
                {"__ndarray__": [shape, dtype name, flat values]})
  item table    int64 offsets of the items' byte counts (item 0 first)

Reader(path)[key] / .key give values, child Readers and numpy arrays (read
on access); Writer(path, tag) mirrors the calls GPAW's writers make
(write(**kw), child(name), add_array(name, shape, dtype) + fill(a),
close())."""
from __future__ import annotations

import json
from typing import Any

import numpy as np

MAGIC = b'- of Ulm'
VERSION = 3


class ULMError(ValueError):
    pass


def _decode_value(v):
    if isinstance(v, dict):
        if '__complex__' in v:
            re, im = v['__complex__']
            return complex(re, im)
        if '__ndarray__' in v:
            shape, dtype, flat = v['__ndarray__']
            dt = np.dtype(dtype)
            if dt.kind == 'c':
                flat = [complex(*x) if isinstance(x, list) else x for x in flat]
            return np.array(flat, dt).reshape(shape)
        return {k: _decode_value(x) for k, x in v.items()}
    if isinstance(v, list):
        return [_decode_value(x) for x in v]
    return v


class Reader:
    """Read access to one item of a ULM file (item 0 by default)."""

    def __init__(self, path, index: int = 0, _data=None, _fd=None):
        if _data is not None:
            self._fd = _fd
            self._data = _data
            return
        self._fd = open(path, 'rb')
        head = self._fd.read(48)
        if len(head) < 48 or head[:8] != MAGIC:
            self._fd.close()
            raise ULMError(f'{path}: not a ULM file')
        self.tag = head[8:24].decode('ascii').rstrip()
        self.format_version, self.nitems, table = (int(x) for x in np.frombuffer(head[24:48], '<i8'))
        if not 0 <= index < self.nitems:
            raise ULMError(f'{path}: item {index} of {self.nitems}')
        self._fd.seek(table + 8 * index)
        (pos,) = np.frombuffer(self._fd.read(8), '<i8')
        self._fd.seek(int(pos))
        (size,) = np.frombuffer(self._fd.read(8), '<i8')
        self._data = json.loads(self._fd.read(int(size)).decode())

    def keys(self):
        return [k[:-1] if k.endswith('.') else k for k in self._data]

    def __contains__(self, key):
        return key in self._data or key + '.' in self._data

    def __getitem__(self, key: str) -> Any:
        if key + '.' in self._data:
            v = self._data[key + '.']
            if 'ndarray' in v:
                shape, dtype, offset = v['ndarray']
                dt = np.dtype(dtype).newbyteorder('<')
                count = int(np.prod(shape)) if len(shape) else 1
                self._fd.seek(int(offset))
                a = np.fromfile(self._fd, dtype=dt, count=count)
                if a.size != count:
                    raise ULMError(f'array {key!r} truncated')
                return a.reshape(shape).astype(dt.newbyteorder('='), copy=False)
            return Reader(None, _data=v, _fd=self._fd)
        if key in self._data:
            return _decode_value(self._data[key])
        raise KeyError(key)

    def __getattr__(self, key: str) -> Any:
        if key.startswith('_'):
            raise AttributeError(key)
        try:
            return self[key]
        except KeyError:
            raise AttributeError(key) from None

    def close(self):
        if self._fd is not None:
            self._fd.close()


def _encode_value(v):
    if isinstance(v, (bool, int, float, str)) or v is None:
        return v
    if isinstance(v, complex):
        return {'__complex__': [v.real, v.imag]}
    if isinstance(v, np.generic):
        return _encode_value(v.item())
    if isinstance(v, np.ndarray):
        flat = [[complex(x).real, complex(x).imag] for x in v.ravel()] if v.dtype.kind == 'c' \
            else v.ravel().tolist()
        return {'__ndarray__': [list(v.shape), v.dtype.name, flat]}
    if isinstance(v, dict):
        return {k: _encode_value(x) for k, x in v.items()}
    if isinstance(v, (list, tuple)):
        return [_encode_value(x) for x in v]
    raise TypeError(f'cannot store {type(v).__name__} in a ULM item')


class Writer:
    """Write one item: header, arrays as they are filled, then (close) the
    item's JSON object and the item table."""

    def __init__(self, path, tag: str = '', _fd=None, _data=None, _root=None):
        self._root = _root or self
        if _fd is not None:
            self._fd, self._data = _fd, _data
            return
        if len(tag) > 16:
            raise ULMError('tag longer than 16 characters')
        self._fd = open(path, 'wb')
        self._fd.write(MAGIC + tag.ljust(16).encode('ascii') + np.zeros(3, '<i8').tobytes())
        self._data = {}
        self._missing = 0
        self._dtype = None

    def _align(self):
        pos = self._fd.tell()
        if pos % 8:
            self._fd.write(b'#' * (8 - pos % 8))
        return self._fd.tell()

    def write(self, **kwargs):
        for name, value in kwargs.items():
            if isinstance(value, np.ndarray) and value.ndim > 0:
                self.add_array(name, value.shape, value.dtype)
                self.fill(value)
            else:
                self._data[name] = _encode_value(value)

    def child(self, name: str) -> 'Writer':
        d = self._data[name + '.'] = {}
        return Writer(None, _fd=self._fd, _data=d, _root=self._root)

    def add_array(self, name: str, shape, dtype=float):
        root = self._root
        if root._missing:
            raise ULMError('the previous array is not filled')
        shape = [int(s) for s in (shape if np.ndim(shape) else (shape,))]
        dt = np.dtype(dtype)
        self._data[name + '.'] = {'ndarray': [shape, dt.name, self._align()]}
        root._missing = int(np.prod(shape)) if shape else 1
        root._dtype = dt

    def fill(self, a):
        root = self._root
        a = np.ascontiguousarray(a, root._dtype.newbyteorder('<'))
        if a.size > root._missing:
            raise ULMError('more data than the array holds')
        root._missing -= a.size
        self._fd.write(a.tobytes())

    def close(self):
        root = self._root
        if root is not self:
            return
        if self._missing:
            raise ULMError('an array is not filled')
        item = self._align()
        blob = json.dumps(self._data).encode()
        self._fd.write(np.array([len(blob)], '<i8').tobytes() + blob)
        table = self._align()
        self._fd.write(np.array([item], '<i8').tobytes())
        self._fd.seek(24)
        self._fd.write(np.array([VERSION, 1, table], '<i8').tobytes())
        self._fd.close()
