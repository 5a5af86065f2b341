"""CPU checks of the drop-in boundary: the C-ABI library loads and exports
every symbol include/sspp.h declares; the command line keeps the reference's
argument handling (src/main.cu:269-321)."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "specseqplusplus_b200", "libsspp.so")
CLI = os.path.join(ROOT, "specseqplusplus_b200", "bin", "specseq++")


def declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sspp_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    assert os.path.exists(LIB), "run __graft_entry__.build() first"
    lib = ctypes.CDLL(LIB)
    names = declared("sspp.h")
    assert len(names) >= 16
    for name in names:
        assert hasattr(lib, name), name


def test_python_mirror_binds_every_symbol():
    from specseqplusplus_b200 import engine

    assert set(declared("sspp.h")) <= set(engine.EXPORTED) | {"sspp_default_params"}


def test_server_without_a_gpu_fails_cleanly():
    from specseqplusplus_b200 import Server, SsppError

    try:
        import torch

        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(SsppError):
        Server()


def test_cli_help_and_argument_errors(tmp_path):
    assert os.path.exists(CLI)
    r = subprocess.run([CLI, "-help"], capture_output=True, text=True)
    assert r.returncode == 0 and "Usage" in r.stdout
    r = subprocess.run([CLI, "a", "b"], capture_output=True, text=True)
    assert r.returncode == 1 and "Invalid number of arguments" in r.stderr
    args = ["in", "out", "text", "ascii", "0", "0", "0", "100", "1.05", "64", "100", "200"]
    r = subprocess.run([CLI] + args, capture_output=True, text=True)
    assert r.returncode == 1 and "Invalid input format" in r.stderr
    args[2], args[3] = "ascii", "xml"
    r = subprocess.run([CLI] + args, capture_output=True, text=True)
    assert r.returncode == 1 and "Invalid output format" in r.stderr


def test_no_oracle_on_product_path():
    # the product never imports, links or runs the oracle
    for dirpath, _, files in os.walk(os.path.join(ROOT, "specseqplusplus_b200")):
        for f in files:
            if f.endswith((".py", ".cu", ".cpp", ".h", ".cuh")):
                text = open(os.path.join(dirpath, f)).read()
                assert "import oracle" not in text and "liboracle" not in text, f


def test_cpp_mirror_header_compiles(tmp_path):
    # the reference-side swap: a main in the reference's style against include/specseq_b200.hpp
    out = tmp_path / "mirror"
    r = subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"),
                        os.path.join(ROOT, "tests", "cpp", "mirror_main.cpp"), "-o", str(out),
                        "-L", os.path.dirname(LIB), "-lsspp", "-Wl,-rpath," + os.path.dirname(LIB)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_c_abi_null_handles(tmp_path):
    # include/sspp.h as plain C99; null handles fail cleanly without a GPU
    out = tmp_path / "abi_null"
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
                        os.path.join(ROOT, "tests", "cpp", "abi_null.c"), "-o", str(out),
                        "-L", os.path.dirname(LIB), "-lsspp", "-Wl,-rpath," + os.path.dirname(LIB)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(out)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr
