"""C++ drop-in front end (include/warpcore/*.cuh): a program written against
warpcore's C++ API -- host bulk methods, device per-key methods called from
user kernels, for_each with a device lambda, status handlers -- compiles and
gives the reference's answers (tests/cpp/dropin_test.cu)."""
import os
import subprocess

import pytest

from tests.cpp import build_dropin

pytestmark = pytest.mark.gpu


def test_cpp_dropin_program():
    exe = build_dropin.build()
    env = dict(os.environ)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "dropin ok" in r.stdout
