"""The C ABI without a GPU: the shared library loads, exports every host
function include/*.h declares, and the status/error paths that need no device
behave as documented (error return vs the prototype's exit(-1)).  Device
functions of nvshmem_device.h / nvshmemx.h are checked by linking a program
that calls each of them against the static library."""
import ctypes
import os
import re
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(REPO, "include")
PKG = os.path.join(REPO, "df-nvshmem-prototype_b200")

DECL = re.compile(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(nvshm\w+|nvstart_pes|nvstop_pes)\s*\(", re.M)


def declared(device: bool):
    names = set()
    for h in sorted(os.listdir(INC)):
        text = open(os.path.join(INC, h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for line in text.splitlines():
            if "#define" in line or "typedef" in line:
                continue
            m = DECL.match(line)
            if not m:
                continue
            is_dev = "__device__" in line
            if is_dev == device:
                names.add(m.group(1))
    return names


def test_shared_library_exports_every_host_symbol():
    from nvshmem_b200._lib import LIB_PATH
    lib = ctypes.CDLL(LIB_PATH)
    names = declared(device=False)
    assert len(names) > 50
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_device_symbols_declared():
    names = declared(device=True)
    for n in ("nvshmem_int_put", "nvshmem_double_get", "nvshmem_int_wait_until", "nvshmem_quiet",
              "nvshmem_float_p", "nvshmem_double_g", "nvshmemx_barrier_all", "nvshmemx_putmem_bulk_block"):
        assert n in names


def _run(code: str, env=None):
    return subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=120,
                          env=env, cwd=REPO)


PRE = ("import sys; sys.path.insert(0, %r); from nvshmem_b200 import _lib as L; lib = L.lib\n"
       % os.path.join(PKG, "python"))


def test_error_mode_exit_matches_prototype():
    # nvshmalloc before start: the prototype prints and calls exit(-1)
    r = _run(PRE + "lib.nvshmalloc(16)\nprint('not reached')")
    assert r.returncode == 255 and "not reached" not in r.stdout
    assert "nvshmalloc before nvstart_pes" in r.stderr


def test_error_mode_return():
    r = _run(PRE + "lib.nvshmemx_set_error_mode(L.ERRORS_RETURN)\n"
             "p = lib.nvshmalloc(16)\nprint(p, lib.nvshmemx_status(), lib.nvshmemx_status())")
    assert r.returncode == 0, r.stderr
    p, st1, st2 = r.stdout.split()
    assert p == "None" and int(st1) == 4 and int(st2) == 0  # ERR_STATE once, then cleared


def test_error_mode_from_environment():
    env = dict(os.environ, NVSHMEM_ERROR_MODE="return")
    r = _run(PRE + "print(lib.nvshmemx_get_error_mode(), lib.nvshmem_ptr(None, 0))", env=env)
    assert r.stdout.split()[0] == "1"


def test_strerror_and_queries_without_start():
    from nvshmem_b200._lib import lib, strerror
    assert strerror(5) == "wait or barrier deadline passed"
    assert lib.nvshmemx_is_started() == 0
    assert lib.nvshmem_n_pes() == 0 and lib.nvshmem_my_pe() == 0


def test_bad_init_arguments_return_codes():
    r = _run(PRE + "lib.nvshmemx_set_error_mode(1)\n"
             "print(lib.nvshmemx_init_attr(0, 1<<20), lib.nvshmemx_init_attr(5000, 1<<20), "
             "lib.nvshmemx_init_attr(2, 0))")
    assert r.stdout.split() == ["1", "1", "1"]


def test_bootstrap_refusals_need_no_device(tmp_path):
    """nvshmemx_init_bootstrap refuses a bad description, and a failing
    allgather callback ends the start with ERR_STATE and leaves no
    rendezvous directory behind (rank 0 made one before the callback)."""
    code = PRE + "\n".join([
        "import ctypes, os",
        "lib.nvshmemx_set_error_mode(1)",
        "AG = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p)",
        "class BS(ctypes.Structure):",
        "    _fields_ = [('rank', ctypes.c_int), ('size', ctypes.c_int), ('allgather', AG), ('ctx', ctypes.c_void_p)]",
        "fail = AG(lambda i, o, n, c: -1)",
        "f = lib.nvshmemx_init_bootstrap",
        "f.argtypes = [ctypes.c_void_p, ctypes.c_size_t]",
        "bad = BS(2, 2, fail, None)",
        "r1 = f(None, 1 << 20)",
        "r2 = f(ctypes.byref(bad), 1 << 20)",
        "r3 = f(ctypes.byref(BS(0, 1, fail, None)), 1 << 20)",
        "print(r1, r2, r3, lib.nvshmemx_is_started(), len(os.listdir(os.environ['TMPDIR'])))",
    ])
    r = _run(code, env=dict(os.environ, TMPDIR=str(tmp_path)))
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.split() == ["1", "1", "4", "0", "0"]


NATIVE = os.path.join(REPO, "tests", "native")


@pytest.mark.skipif(subprocess.run(["which", "nvcc"], capture_output=True).returncode != 0, reason="no nvcc")
def test_every_device_function_links_against_static_lib(tmp_path):
    src = os.path.join(NATIVE, "api_all.cu")
    out = tmp_path / "api_all"
    lib = os.path.join(PKG, "lib")
    r = subprocess.run(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-rdc=true", "-I", INC, src,
                        "-o", str(out), "-L", lib, "-lnvshmem", "-L/usr/local/cuda/lib64/stubs", "-lcuda"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-3000:]
    assert out.exists()


@pytest.mark.skipif(subprocess.run(["which", "nvcc"], capture_output=True).returncode != 0, reason="no nvcc")
def test_every_device_function_links_with_device_lto(tmp_path):
    """The static library also carries LTO IR: an application compiled with
    code=lto_100a and linked with -dlto gets the device calls inlined."""
    src = os.path.join(NATIVE, "api_all.cu")
    obj, out = tmp_path / "api_all.o", tmp_path / "api_all_lto"
    lib = os.path.join(PKG, "lib")
    r = subprocess.run(["nvcc", "-gencode", "arch=compute_100a,code=lto_100a", "-rdc=true", "-I", INC, "-c", src,
                        "-o", str(obj)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-3000:]
    r = subprocess.run(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-dlto", "-rdc=true", str(obj),
                        "-o", str(out), "-L", lib, "-lnvshmem", "-L/usr/local/cuda/lib64/stubs", "-lcuda"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-3000:]
    assert out.exists()


def _reference_readable():
    r = subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle", "ref_build"), "have-ref"],
                       capture_output=True, text=True)
    return r.returncode == 0


@pytest.mark.skipif(subprocess.run(["which", "nvcc"], capture_output=True).returncode != 0, reason="no nvcc")
@pytest.mark.skipif(not _reference_readable(), reason="the reference sources are not on this machine")
def test_reference_microbenchmarks_build_unchanged_against_this_library():
    """The prototype's two microbenchmarks (microbench/shmem_latency.cu and
    microbench/shmem_sync_latency.cu), compiled as they are with this
    library's nvshmem.h / nvshmem_device.h and linked with its libnvshmem.a
    (oracle/ref_build, target `compat`; the project's MPI subset stands in for
    MPI).  They are not run: their two ranks spin on each other from separate
    processes, which one GPU does not guarantee to run together."""
    ref_build = os.path.join(REPO, "oracle", "ref_build")
    deps = subprocess.run(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-rdc=true", "-I", INC, "-I",
                           ref_build, "-M", "-x", "cu", "-"], input='#include "nvshmem.h"\n#include "nvshmem_device.h"\n',
                          capture_output=True, text=True, timeout=300)
    assert deps.returncode == 0 and os.path.join(INC, "nvshmem.h") in deps.stdout
    r = subprocess.run(["make", "-B", "-C", ref_build, "compat"], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-3000:]
    for name in ("compat_shmem_latency", "compat_shmem_sync_latency"):
        assert os.path.exists(os.path.join(REPO, "oracle", "_ref", name))
