"""The tuning table round trip (JSON -> library -> cm_tuning_get), no GPU."""
import json

from contactmechanics_b200 import Autotune, _lib


def test_tuning_table_round_trip(tmp_path):
    L = _lib.load_library()
    table = {"tiles": {"fp32": {"96": 4096, "128": 1024}, "fp64": {"96": 512}},
             "threads": {"fp32": 128, "fp64": 512}}
    path = tmp_path / "t.json"
    Autotune.save(table, str(path))
    Autotune.apply(Autotune.load(str(path)))
    import ctypes
    e, t = ctypes.c_int(), ctypes.c_int()
    assert L.cm_tuning_get(_lib.CM_FP32, 96, ctypes.byref(e), ctypes.byref(t)) == 0
    assert (e.value, t.value) == (4096, 128)
    assert L.cm_tuning_get(_lib.CM_FP64, 96, ctypes.byref(e), ctypes.byref(t)) == 0
    assert (e.value, t.value) == (512, 512)
    assert L.cm_tuning_get(_lib.CM_FP64, 200, ctypes.byref(e), ctypes.byref(t)) == 0
    assert e.value == 2048  # default for lengths without an entry
    assert L.cm_tuning_set_batch_threads(_lib.CM_FP32, 100) == _lib.CM_ERR_ARG
    Autotune.clear(lengths=(96, 128))
    assert L.cm_tuning_get(_lib.CM_FP32, 96, ctypes.byref(e), ctypes.byref(t)) == 0
    assert (e.value, t.value) == (2048, 256)
    if (Autotune.DEFAULT_TABLE and __import__("os").path.exists(Autotune.DEFAULT_TABLE)):
        shipped = Autotune.load()
        assert set(shipped["tiles"]) == {"fp32", "fp64"}
        assert all(int(v) in (512, 1024, 2048, 4096) for d in shipped["tiles"].values()
                   for v in d.values())
