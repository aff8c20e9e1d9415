"""C-ABI surface on CPU: the library loads, exports every function include/hidem_b200.h
declares, mirrors the sample defaults, and fails cleanly without a GPU."""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import pytest

from hidem_b200 import abi

HEADER = Path(__file__).resolve().parents[1] / "include" / "hidem_b200.h"


def declared_functions() -> list[str]:
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(hidem_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = abi.load()
    names = declared_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # and the ctypes prototypes cover the header
    assert set(names) <= set(abi.EXPORTED)


def test_abi_version_and_struct_sizes():
    lib = abi.load()
    assert lib.hidem_abi_version() == 1
    # C layout of the params struct: 22 doubles + 2x3 doubles + 2x3 int32 + ...
    assert C.sizeof(abi.HidemParticleSoA) == 16 * 8
    assert C.sizeof(abi.HidemLinkSoA) == 13 * 8


def test_defaults_are_the_meshblock_sample_defaults():
    p = abi.default_params()
    # HiDEM/MeshBlock/MainMeshBlock.cpp:69-102, HiDEMLib/HiDEMLib.h:744-745
    assert p.dt == 0.0001 and p.scale == 1.0 and p.E == 1e9 and p.beamWidth == 0.6
    assert p.damping == 1000.0 and p.dampingRotation == 1000.0
    assert p.maxLoad == 0.35 and p.bendBreak == 0.35 and p.breakTime == 10.0
    assert p.rhoIce == 910.0 and p.rhoWater == 1030.0 and p.g == 9.81
    assert p.maxVel == 20 and p.maxRot == 5 and p.searchDistanceScale == 1.4
    assert p.gridRegenInterval == -1 and p.firstBalanceTimestep == 2000
    assert p.precision == abi.PREC_MIXED


def test_create_rejects_bad_params_without_touching_cuda():
    lib = abi.load()
    p = abi.default_params(precision=7)
    h = C.c_void_p()
    assert lib.hidem_create(C.byref(p), 0, C.byref(h)) == 1  # HIDEM_ERR_ARG
    assert b"precision" in lib.hidem_create_error()
    p = abi.default_params(dt=-1.0)
    assert lib.hidem_create(C.byref(p), 0, C.byref(h)) == 1
    assert not h.value


def test_create_without_device_is_a_status_not_a_crash():
    from conftest import cuda_available
    if cuda_available():
        pytest.skip("a GPU is present")
    lib = abi.load()
    p = abi.default_params()
    h = C.c_void_p()
    st = lib.hidem_create(C.byref(p), 0, C.byref(h))
    assert st == 2  # HIDEM_ERR_CUDA
    assert not h.value
    assert lib.hidem_create_error()


def test_null_context_calls_return_arg_error():
    lib = abi.load()
    assert lib.hidem_step(None, 1) == 1
    assert lib.hidem_grid_service(None) == 1
    assert lib.hidem_compute_forces(None) == 1
    assert lib.hidem_last_error(None) == b"null context"
    # the slab decomposition hooks
    import ctypes as C
    import numpy as np
    mx, lo, hi = np.zeros(3), np.zeros(3), np.ones(3)
    flag = C.c_int32()
    assert lib.hidem_grid_service_local(None, mx.ctypes.data, C.byref(flag)) == 1
    assert lib.hidem_grid_service_decide(None, mx.ctypes.data, C.byref(flag)) == 1
    assert lib.hidem_local_bounds(None, lo.ctypes.data, hi.ctypes.data) == 1
    assert lib.hidem_regenerate_frame(None, lo.ctypes.data, hi.ctypes.data) == 1
    assert lib.hidem_set_halo_exchange(None, None, 0, None, 0) == 1
    assert lib.hidem_pack_halo_forces(None, None) == 1
    assert lib.hidem_unpack_halo_forces(None, None) == 1


def test_soa_checks_dtypes_and_sizes():
    p = abi.empty_particles(4, abi.PREC_MIXED)
    abi.particle_soa(p, abi.PREC_MIXED, 4)
    with pytest.raises(TypeError):
        abi.particle_soa(p, abi.PREC_FP64, 4)
    with pytest.raises(ValueError):
        abi.particle_soa(p, abi.PREC_MIXED, 5)


def test_cpp_adapter_compiles_and_links(tmp_path):
    """include/hidem_b200.hpp (the HiDEMLib-shaped C++ binding) compiles against the
    header and links against the library; without a GPU, construction throws a status."""
    import shutil
    import subprocess
    from conftest import cuda_available
    gxx = "/usr/bin/g++" if Path("/usr/bin/g++").exists() else shutil.which("g++")
    if not gxx:
        pytest.skip("no C++ compiler")
    root = Path(__file__).resolve().parents[1]
    src = tmp_path / "adapter.cpp"
    src.write_text(r'''
#include "hidem_b200.hpp"
#include <cstdio>
int main() {
    hidem_params p;
    hidem_params_default(&p);
    try {
        hidem::HiDEMLibB200 lib(p, 0);
        std::printf("created step=%lld\n", (long long)lib.getCurrentTimestep());
        lib.setBedMaps(nullptr, nullptr);
        lib.setCollisionMesh(nullptr);
        lib.setStepKernel(HIDEM_STEP_KERNEL_AUTO);
        if (lib.getStats().num_particles > 0) {
            lib.computePartForce(hidem::NeighForceFunc{1e4, 0, 0, 1, 1, 1e9},
                                 hidem::LinkForceFunc{1e4, 1, 1, 1e9, 1, 1, 5e8});
            lib.linkUpdate(hidem::LinkBreakFunc{0.01, 5e-4});
        }
        double kt = 0, kr = 0, vm = 0;
        if (lib.getStats().num_particles > 0) lib.kineticEnergy(kt, kr, vm);
    } catch (const hidem::Error &e) {
        std::printf("status=%d\n", (int)e.status);
    }
    return 0;
}
''')
    exe = tmp_path / "adapter"
    r = subprocess.run([gxx, "-std=c++17", f"-I{root / 'include'}", str(src), "-o", str(exe),
                        f"-L{root / 'hidem_b200'}", "-lhidem_b200",
                        f"-Wl,-rpath,{root / 'hidem_b200'}"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0
    if not cuda_available():
        assert "status=2" in out.stdout


def test_device_view_struct_matches_the_header(tmp_path):
    """hidem_device_view's size and field offsets as a C compiler lays them out."""
    import shutil
    import subprocess
    gcc = shutil.which("gcc") or "/usr/bin/gcc"
    src = tmp_path / "v.c"
    src.write_text('#include <stddef.h>\n#include <stdio.h>\n#include "hidem_b200.h"\n'
                   'int main(void){printf("%zu %zu %zu %zu\\n", sizeof(hidem_device_view),'
                   ' offsetof(hidem_device_view, end_ct), offsetof(hidem_device_view, event_capacity),'
                   ' offsetof(hidem_device_view, stream)); return 0;}\n')
    exe = tmp_path / "v"
    r = subprocess.run([gcc, f"-I{HEADER.parent}", str(src), "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()
    V = abi.HidemDeviceView
    assert [int(x) for x in out] == [C.sizeof(V), V.end_ct.offset, V.event_capacity.offset, V.stream.offset]


def test_iterate_header_compiles_for_sm100a(tmp_path):
    """include/hidem_b200_iterate.cuh with a caller's functors (tests/iterate_harness.cu)
    cross-compiles for sm_100a (the GPU tests run it)."""
    import shutil
    import subprocess
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(nvcc).exists():
        pytest.skip("no nvcc")
    src = Path(__file__).with_name("iterate_harness.cu")
    r = subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-O1",
                        "-fmad=false", f"-I{HEADER.parent}", "-c", str(src), "-o", str(tmp_path / "h.o")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
