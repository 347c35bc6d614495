"""Persistence of the autotuners' launch choices.

The stencil launchers time their tile variants / row layouts on the first
launch of every new shape (outside stream capture) and keep the fastest in
process memory.  ``save(path)`` writes those choices to a JSON file and
``load(path)`` merges them into a new process, so that it launches the
tuned layouts at once instead of timing them again.  Records carry the
device name and SM count; a file from another device is refused.

With the environment variable ``GPW_TUNE_CACHE`` set to a path, the first
load of the library merges that file (when it exists) and the process saves
its choices there at exit.
"""
import ctypes
import json
import os

from . import _lib

FORMAT = 'gpwgrid-tune-json 1'


def export_records():
    """The tuners' records as text (gpw_tune_export)."""
    lib = _lib.load()
    need = ctypes.c_int64()
    _lib.check(lib.gpw_tune_export(None, 0, ctypes.byref(need)))
    buf = ctypes.create_string_buffer(int(need.value))
    _lib.check(lib.gpw_tune_export(buf, int(need.value), ctypes.byref(need)))
    return buf.value.decode()


def import_records(text):
    """Merge records; returns how many were taken (gpw_tune_import)."""
    lib = _lib.load()
    n = ctypes.c_int()
    _lib.check(lib.gpw_tune_import(text.encode(), ctypes.byref(n)))
    return n.value


def save(path):
    with open(path + '.tmp', 'w') as f:
        json.dump({'format': FORMAT, 'records': export_records()}, f)
    os.replace(path + '.tmp', path)


def load(path):
    with open(path) as f:
        d = json.load(f)
    if d.get('format') != FORMAT:
        raise ValueError('%s is not a gpwgrid tuning file' % path)
    return import_records(d['records'])


def _auto(path):
    import atexit
    if os.path.exists(path):
        try:
            load(path)
        except Exception:   # a cache from another device: tune afresh
            pass

    def _save():
        try:
            save(path)
        except Exception:
            pass
    atexit.register(_save)
