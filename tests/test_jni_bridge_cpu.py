"""The JNI bridge compiled and called without a JDK or a GPU: the five
Java_br_unb_cic_tdp_base_GPUSortingSearch_* symbols (jni_sorter.cu:25-150) through a stand-in
VM (tests/jni).  Without a device every call that reaches CUDA fails, so this covers the
argument checks and the RuntimeException texts of the reference (sorting_search.cu:707-715,
jni_sorter.cu:16-23), plus void calls that must not throw."""
import numpy as np

import jni_harness as J

R1375 = float(np.float32(2) / np.float32(1.375))
PI7 = [0, 4, 5, 6, 3, 1, 2]
SPI7 = [3, 5, 6, 4, 1, 2, 0]


def test_bridge_error_paths_without_a_device(tmp_path, native_lib):
    exe = J.build(str(tmp_path))
    out = J.run(exe, [
        "init 1 1 1048576 1048576",
        J.search_line(0, R1375, 4, True, 3, list(range(64)), list(range(64))),
        J.search_line(0, R1375, 0, True, 3, PI7, SPI7),
        J.search_line(0, R1375, 16, True, 3, PI7, SPI7),
        J.search_line(5, R1375, 4, True, 3, PI7, SPI7),
        J.search_line(0, R1375, 4, True, 3, PI7, SPI7[:-1], mismatch=True),
        "cancel 3",
        "destroy",
        "destroy",
        J.filter_line(False, 64, [0, 1, 2], [0, 1, 2]),
    ], str(tmp_path))
    assert [o["exception"] for o in out] == [
        "initSlots: no CUDA device",
        "performGpuSortingSearch: n exceeds MAX_N",
        "performGpuSortingSearch: invalid maximumDepth",
        "performGpuSortingSearch: invalid maximumDepth",
        "invalid slot",
        "performGpuSortingSearch: inconsistent input sizes",
        None,  # cancelSort has no failure path (jni_sorter.cu:106-109)
        None,  # destroySlots is idempotent
        None,
        "n exceeds PI_FILTER_MAX_N",
    ]
    # a method that throws returns null, as the reference's JNI layer does (jni_sorter.cu:103, 149)
    assert all(o["null_result"] for o in out if o["exception"] and o["call"].startswith(("search", "filter")))
