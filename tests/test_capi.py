"""CPU: the C-ABI library loads, exports every entry point declared in
include/bipp_b200.h, and fails loudly (no CPU fallback) without a GPU."""
import ctypes as C
import os
import re

import pytest

from conftest import ROOT


def _declared():
    src = open(os.path.join(ROOT, "include", "bipp_b200.h")).read()
    return sorted(set(re.findall(r"BIPP_B200_EXPORT\s+[\w\s\*]+?\b(bipp_\w+)\s*\(", src)))


def test_header_declares_entry_points():
    names = _declared()
    for n in ("bipp_eigh_gram_s", "bipp_eigh_gram_d", "bipp_nufft_add_s", "bipp_nufft_get_image",
              "bipp_nuft_sum_s", "bipp_image_synthesis", "bipp_pipeline_process", "bipp_domain_partition_grid_s"):
        assert n in names


def test_library_exports_every_declared_symbol():
    from bipp_b200 import _lib

    lib = _lib.load()
    for n in _declared():
        assert hasattr(lib, n), n
        assert n in _lib.SIGNATURES, n


def test_library_in_tree_and_build_recipe_targets_only_sm100a():
    """The library is built in the source tree, and the build recipe compiles and links
    device code for sm_100a alone (no other -gencode target, no PTX fallback)."""
    from bipp_b200 import _lib, build

    assert os.path.dirname(_lib.LIB_PATH) == os.path.join(ROOT, "bipp_b200")
    assert os.path.getsize(_lib.LIB_PATH) > 100_000
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
    assert all("arch=" not in f and "-arch" not in f for f in build._flags() if f not in build.ARCH)


def test_no_cpu_processing_unit():
    import bipp_b200 as bipp

    with pytest.raises(bipp.BippError):
        bipp.Context("CPU")


def test_context_without_gpu_raises_gpu_support_error():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import bipp_b200 as bipp

    with pytest.raises(bipp.GPUError):
        bipp.Context("GPU")


def test_error_message_plumbing():
    from bipp_b200 import _lib

    lib = _lib.load()
    h = C.c_void_p()
    rc = lib.bipp_ctx_create(1, C.byref(h))  # CPU rejected
    assert rc == 3
    assert b"CPU" in lib.bipp_last_error()


def test_null_handles_are_rejected_without_a_gpu():
    """Every entry point checks its handle and pointers before any device work: null
    handles give BIPP_INVALID_POINTER_ERROR (4) or BIPP_INVALID_HANDLE_ERROR (5) with a
    message, and destroying a null handle succeeds (as deleting a null object)."""
    from bipp_b200 import _lib

    lib = _lib.load()
    for name, argtypes in _lib.SIGNATURES.items():
        if name in ("bipp_last_error", "bipp_kernel_launch_count", "bipp_rank_mlp_num_params", "bipp_tuning_reset"):
            continue
        args = []
        for t in argtypes:
            if t in (C.c_float, C.c_double):
                args.append(t(2.0))
            elif t in (C.c_int, C.c_size_t):
                args.append(t(4))
            else:
                args.append(None)
        rc = getattr(lib, name)(*args)
        if name.endswith("_destroy"):
            assert rc == 0, name
        else:
            assert rc in (4, 5), (name, rc)
            assert b"null" in lib.bipp_last_error(), name


def test_cxx_shell_host_checks(tmp_path):
    """The bipp C++ API shell (include/bipp/*.hpp) compiles and links against the
    library with g++, and its host-side behaviour holds without a GPU: exception types
    and codes, the CPU processing unit rejected, GPUSupportError for a GPU context
    without a device, Communicator::world() (tests/cxx/shell_cpu_check.cpp)."""
    import subprocess

    import torch

    exe = tmp_path / "shell_cpu_check"
    libdir = os.path.join(ROOT, "bipp_b200")
    subprocess.run(["g++", "-std=c++17", "-O1", os.path.join(ROOT, "tests", "cxx", "shell_cpu_check.cpp"),
                    "-I" + os.path.join(ROOT, "include"), "-I/usr/local/cuda/include", "-L" + libdir,
                    "-lbipp_b200", "-Wl,-rpath," + libdir, "-o", str(exe)], check=True)
    args = [str(exe)] + ([] if torch.cuda.is_available() else ["no-gpu"])
    r = subprocess.run(args, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr


def test_pybipp_surface():
    """The names and members of pybipp (python/pybipp.cpp:285-493) that the reference's
    Python pipeline uses exist with the same call shapes (no device needed)."""
    import inspect

    import bipp_b200 as bipp
    from bipp_b200 import (Context, NufftSynthesisOptions, Partition, communicator, config,  # noqa: F401
                           eigh, eigh_gram, gram_matrix, image_synthesis)

    opt = NufftSynthesisOptions()
    for m in ("set_tolerance", "set_sample_batch_size", "set_local_uvw_partition", "set_normalize_image",
              "set_apply_scaling", "set_precision"):
        assert callable(getattr(opt, m)), m
    for a in ("tolerance", "sample_batch_size", "local_uvw_partition", "normalize_image", "apply_scaling",
              "precision"):
        assert hasattr(opt, a), a
    assert opt.set_precision("double").precision == "double"
    with pytest.raises(bipp.InvalidParameterError):
        opt.set_precision("half")
    assert Partition.grid([2, 3, 4]).dims == (2, 3, 4)
    assert Partition.auto().method == "auto" and Partition.none().method == "none"
    assert isinstance(Context.processing_unit, property)
    assert list(inspect.signature(Context).parameters)[:2] == ["pu", "comm"]
    assert list(inspect.signature(eigh_gram).parameters)[:4] == ["wl", "s", "w", "xyz"]
    assert list(inspect.signature(eigh).parameters)[:3] == ["wl", "s", "w"]
    assert list(inspect.signature(image_synthesis).parameters)[:6] == ["ctx", "opt", "dataset", "selection",
                                                                       "image_prop", "image_file_name"]
    assert all(hasattr(config, f) for f in ("cuda", "rocm", "umpire", "omp", "mpi"))
    assert (communicator.local().rank, communicator.local().size) == (0, 1)


def test_tuning_table_without_a_gpu(tmp_path):
    """The autotuner's table of launch parameters (no device needed): defaults, candidate
    checks, save / load round trip, the environment file, reset."""
    import bipp_b200 as bipp

    bipp.tuning_reset()
    assert bipp.tuning_get("spread.items_cap") == 2048 and bipp.tuning_get("hetrd.threads") == 0
    desc = bipp.tuning_describe()
    assert set(desc) == {"spread.items_cap", "spread.operands", "spread.stages", "spread.ctas_per_sm", "spread.schedule",
                         "hetrd.threads", "hetrd.ctas_pct", "tridiag.threads", "bt.columns", "vv.ctas_per_sm", "direct.ctas_per_sm", "nufft.fft",
                         "nufft.grid_per_1024"}
    assert desc["spread.items_cap"]["candidates"] == [2048, 4096, 8192]
    with pytest.raises(bipp.InvalidParameterError):
        bipp.tuning_set("spread.items_cap", 1000)
    with pytest.raises(bipp.InvalidParameterError):
        bipp.tuning_get("no.such.parameter")
    bipp.tuning_set("spread.items_cap", 8192)
    bipp.tuning_set("hetrd.threads", 512)
    f = tmp_path / "tune.txt"
    bipp.tuning_save(str(f))
    bipp.tuning_reset()
    assert bipp.tuning_get("spread.items_cap") == 2048
    bipp.tuning_load(str(f))
    assert bipp.tuning_get("spread.items_cap") == 8192 and bipp.tuning_get("hetrd.threads") == 512
    bad = tmp_path / "bad.txt"
    bad.write_text("vv.ctas_per_sm 7\n")
    with pytest.raises(bipp.InvalidParameterError):
        bipp.tuning_load(str(bad))
    bipp.tuning_reset()


def test_cxx_shell_image_reduction_over_three_ranks(tmp_path):
    """The C++ API's Communicator::world() sums float arrays of three ranks (processes)
    into rank 0 over TCP, exactly; custom() runs the caller's reduction
    (tests/cxx/reduce_check.cpp). No GPU is needed."""
    import socket
    import subprocess

    exe = tmp_path / "reduce_check"
    libdir = os.path.join(ROOT, "bipp_b200")
    subprocess.run(["g++", "-std=c++17", "-O1", os.path.join(ROOT, "tests", "cxx", "reduce_check.cpp"),
                    "-I" + os.path.join(ROOT, "include"), "-I/usr/local/cuda/include", "-L" + libdir,
                    "-lbipp_b200", "-Wl,-rpath," + libdir, "-o", str(exe)], check=True)
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    procs = []
    for r in range(3):
        env = dict(os.environ, RANK=str(r), WORLD_SIZE="3", MASTER_ADDR="127.0.0.1", BIPP_B200_REDUCE_PORT=str(port),
                   BIPP_B200_REDUCE_TIMEOUT="60")
        procs.append(subprocess.Popen([str(exe)], env=env, stderr=subprocess.PIPE, text=True))
    for p in procs:
        _, err = p.communicate(timeout=120)
        assert p.returncode == 0, err
