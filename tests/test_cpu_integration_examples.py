"""The code examples of the integration guide still match the headers: the
MPI bootstrap in C compiles against include/ (with a stand-in mpi.h: MPI is
not installed here), and the ctypes example is valid Python."""
import os
import re
import subprocess

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GUIDE = os.path.join(REPO, "INTEGRATION.md")

MPI_STANDIN = """typedef int MPI_Comm;
typedef int MPI_Datatype;
#define MPI_BYTE 1
#define MPI_SUCCESS 0
int MPI_Allgather(const void *, int, MPI_Datatype, void *, int, MPI_Datatype, MPI_Comm);
int MPI_Comm_rank(MPI_Comm, int *);
int MPI_Comm_size(MPI_Comm, int *);
"""


def _blocks(lang):
    with open(GUIDE) as f:
        return re.findall(r"```" + lang + r"\n(.*?)```", f.read(), re.S)


@pytest.mark.skipif(subprocess.run(["which", "gcc"], capture_output=True).returncode != 0, reason="no gcc")
def test_c_examples_compile_against_the_headers(tmp_path):
    blocks = _blocks("c")
    assert blocks
    (tmp_path / "mpi.h").write_text(MPI_STANDIN)
    for k, code in enumerate(blocks):
        src = tmp_path / f"example{k}.c"
        src.write_text(code)
        r = subprocess.run(["gcc", "-fsyntax-only", "-std=c11", "-Wall", "-Werror", "-I", os.path.join(REPO, "include"),
                            "-I", str(tmp_path), "-I", "/usr/local/cuda/include", str(src)],
                           capture_output=True, text=True, timeout=120)
        assert r.returncode == 0, r.stderr[-2000:]


def test_python_examples_parse():
    blocks = _blocks("python")
    assert blocks
    for k, code in enumerate(blocks):
        compile(code, f"INTEGRATION.md python block {k}", "exec")


def test_cgo_example_uses_declared_names():
    """Go is not installed here: check instead that every C.name the cgo
    example calls or names is declared in the headers it includes."""
    blocks = _blocks("go")
    assert blocks
    names = set(re.findall(r"\bC\.([A-Za-z_][A-Za-z0-9_]*)", "".join(blocks)))
    builtin = {"int", "float", "GoString", "char", "size_t", "longlong", "ulonglong"}
    headers = ""
    for h in ("nvshmem.h", "nvshmemx.h", "nvshmemx_batch.h"):
        with open(os.path.join(REPO, "include", h)) as f:
            headers += f.read()
    missing = [n for n in sorted(names - builtin) if not re.search(r"\b" + n + r"\b", headers)]
    assert not missing, missing
    assert "nvshmemx_batch_submit" in names and "nvshmemx_last_error_string" in names
