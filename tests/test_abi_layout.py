"""The Python binding's mirrors of the C-ABI structs (ctypes Structures and numpy dtypes) have the
header's field names, offsets and sizes: a C program compiled against include/curfil_b200.h prints
offsetof/sizeof for every mirrored field, and each must equal the binding's."""
import ctypes
import os
import shutil
import subprocess

import pytest

import curfil_b200 as cf

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

MIRRORS = {
    "cf_sample": cf.SAMPLE_DTYPE,
    "cf_split": cf.SPLIT_DTYPE,
    "cf_train_config": cf.TrainConfig,
    "cf_eval_tuning": cf.EvalTuning,
    "cf_server_config": cf.ServerConfig,
    "cf_request_stats": cf.RequestStats,
    "cf_refiner_config": cf.RefinerConfig,
}


def _python_layout(mirror):
    """[(field, offset)], size of a ctypes Structure or numpy structured dtype."""
    if isinstance(mirror, type) and issubclass(mirror, ctypes.Structure):
        return [(name, getattr(mirror, name).offset) for name, *_ in mirror._fields_], ctypes.sizeof(mirror)
    return [(name, mirror.fields[name][1]) for name in mirror.names], mirror.itemsize


def test_binding_structs_match_the_header(tmp_path):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "curfil_b200.h"', "int main(void) {"]
    expected = []
    for struct, mirror in MIRRORS.items():
        fields, size = _python_layout(mirror)
        lines.append('printf("%s sizeof %%zu\\n", sizeof(%s));' % (struct, struct))
        expected.append("%s sizeof %d" % (struct, size))
        for name, off in fields:
            lines.append('printf("%s.%s %%zu\\n", offsetof(%s, %s));' % (struct, name, struct, name))
            expected.append("%s.%s %d" % (struct, name, off))
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    r = subprocess.run([cc, "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, "a mirrored field is missing from the header:\n" + r.stderr
    got = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    assert [g for g in got if g] == expected
