"""The Python bindings agree with include/risgraph_b200.h: every struct the
ctypes facade mirrors has the C size and field offsets (checked by compiling
a probe against the header with the host compiler), and the option names map
to the header's rg_option values.  No GPU is needed."""
import ctypes
import os
import re
import shutil
import subprocess

import pytest

import risgraph_b200 as rg

INCLUDE = os.path.join(os.path.dirname(os.path.dirname(__file__)), "include")
HEADER = os.path.join(INCLUDE, "risgraph_b200.h")

# C struct -> its ctypes mirror; C record -> its numpy dtype
STRUCTS = {"rg_tune_report": rg.TuneReport, "rg_server_stats": rg.ServerStats, "rg_load_config": rg.LoadConfig,
           "rg_load_result": rg.LoadResult, "rg_frontend_stats": rg.FrontendStats}
DTYPES = {"rg_edge": rg.EDGE_DTYPE, "rg_request": rg.REQUEST_DTYPE, "rg_completion": rg.COMPLETION_DTYPE,
          "rg_client_update_request": rg.CLIENT_REQUEST_DTYPE, "rg_client_update_response": rg.CLIENT_RESPONSE_DTYPE,
          "rg_wal_record": rg.WAL_RECORD_DTYPE}


def _mirror(name):
    return STRUCTS[name]


@pytest.fixture(scope="module")
def c_layout(tmp_path_factory):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no host C compiler")
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "risgraph_b200.h"', "int main(void) {"]
    for name in STRUCTS:
        lines.append(f'  printf("{name} size %zu\\n", sizeof({name}));')
        for f, _ in _mirror(name)._fields_:
            lines.append(f'  printf("{name} {f} %zu\\n", offsetof({name}, {f}));')
    for name, dt in DTYPES.items():
        lines.append(f'  printf("{name} size %zu\\n", sizeof({name}));')
        for f in dt.names:
            lines.append(f'  printf("{name} {f} %zu\\n", offsetof({name}, {f}));')
    lines += ["  return 0;", "}"]
    d = tmp_path_factory.mktemp("layout")
    src, exe = d / "probe.c", d / "probe"
    src.write_text("\n".join(lines) + "\n")
    subprocess.run([cc, "-std=c11", "-I" + INCLUDE, str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    res = {}
    for ln in out.splitlines():
        s, f, v = ln.split()
        res[(s, f)] = int(v)
    return res


@pytest.mark.parametrize("name", sorted(STRUCTS))
def test_ctypes_structs_match_header(c_layout, name):
    m = _mirror(name)
    assert ctypes.sizeof(m) == c_layout[(name, "size")], name
    for f, _ in m._fields_:
        assert getattr(m, f).offset == c_layout[(name, f)], (name, f)


@pytest.mark.parametrize("name", sorted(DTYPES))
def test_numpy_records_match_header(c_layout, name):
    dt = DTYPES[name]
    assert dt.itemsize == c_layout[(name, "size")], name
    for f in dt.names:
        assert dt.fields[f][1] == c_layout[(name, f)], (name, f)


def test_option_names_match_header_enum():
    text = open(HEADER).read()
    body = re.search(r"typedef enum \{([^}]*)\} rg_option;", text).group(1)
    header = {k: int(v) for k, v in re.findall(r"RG_OPT_(\w+)\s*=\s*(\d+)", body)}
    py = dict(rg.Graph.OPTIONS)
    # every Python name maps to the header's value of the same knob
    names = {"dense_pull": "DENSE_PULL", "dense_div": "DENSE_DIV", "lbs_min": "LBS_MIN",
             "bfs_bottom_up": "BFS_BOTTOM_UP", "recompute_min": "RECOMPUTE_MIN", "bu_div": "BFS_BU_DIV",
             "pull_div": "PULL_DIV", "tiny_edges": "TINY_EDGES", "pull_split": "PULL_SPLIT",
             "max_levels": "MAX_LEVELS", "pull_groups": "PULL_GROUPS",
             "fused_max": "FUSED_MAX", "phase_trace": "PHASE_TRACE", "inline_max": "INLINE_MAX", "cluster_edges": "CLUSTER_EDGES"}
    assert set(py) == set(names), set(py) ^ set(names)
    for k, v in py.items():
        assert header[names[k]] == v, k
    assert set(header) == set(names.values())
    # the tuner report has room for every option
    assert max(header.values()) < len(_mirror("rg_tune_report")().options)
