"""Child process for test_harness_matches_unmodified_cal_gso_tasks_cpu: runs the reference's
unmodified cal_gso_tasks_cpu (via oracle/_ref) from a fresh process, so that its fork() happens
before any OpenMP thread pool exists, and prints the reference's stdout."""
import ctypes as C
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

import sparkledock_b200 as sd  # noqa: E402
from oracle_bind import OracleSystem, ref  # noqa: E402

cx = sd.SyntheticComplex(757, 481, 4, 200, seed=7)
tables = sd.synthetic_tables(3)
osys = OracleSystem(cx, tables, cr_math=0)
pos0 = np.ascontiguousarray(cx.poses)
buf = C.create_string_buffer(1 << 20)
rc = ref().ref_run_cal_gso_tasks_cpu(osys.ptr, pos0.ctypes.data_as(C.POINTER(C.c_double)), 2, buf, 1 << 20)
sys.stdout.write(f"RC {rc}\n")
sys.stdout.write(buf.value.decode())
