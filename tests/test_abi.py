"""CPU checks of the C ABI: the library loads, exports every function that
include/*.h declares, the ctypes mirrors have the header's layouts, and the
host-side math (defaults, derived values, lookup tables, density error
factor) matches the oracle. No device work is done here."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
INCLUDE = os.path.join(ROOT, "include")


def declared_functions(headers=("upf.h",)):
    names = set()
    for f in headers:
        src = open(os.path.join(INCLUDE, f)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b([a-zA-Z_]\w*)\s*\(", src, flags=re.M):
            name = m.group(1)
            if name in ("if", "for", "while", "return", "sizeof", "defined"):
                continue
            names.add(name)
    return names


def test_library_exports_every_declared_function(upf_lib):
    lib = upf_lib.lib()
    names = declared_functions()
    assert "upf_create" in names and "upf_step" in names
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_compat_library_exports_every_declared_function(upf_lib):
    """include/upf_compat.h (the reference's own entry points) against
    libupf_compat.so; CopyParticleDataHostToDevice is compiled by the caller
    (compat/upf_compat_particles.cpp reads the caller's particle class)."""
    assert sorted(f for f in os.listdir(INCLUDE) if f.endswith(".h")) == ["upf.h", "upf_compat.h"]
    lib = C.CDLL(os.path.join(os.path.dirname(upf_lib.LIBPATH), "libupf_compat.so"))
    names = declared_functions(("upf_compat.h",)) - {"CopyParticleDataHostToDevice"}
    assert {"ParticlePhysicsOnDevicePCISPH", "CopyParticlesCUDA", "FreeDeviceArrays", "RadixSort"} <= names
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_struct_layouts_match_header(upf_lib, tmp_path):
    from unifiedparticleframeworkcuda_b200._abi import UpfLaunchConfig, UpfParams, UpfPhaseTimes, UpfStepStats
    src = tmp_path / "sz.c"
    src.write_text('#include "upf.h"\n#include <stdio.h>\n#include <stddef.h>\n'
                   'int main(){printf("%zu %zu %zu %zu %zu %zu %zu %zu\\n", sizeof(upf_params), sizeof(upf_step_stats),'
                   ' offsetof(upf_params, scales), offsetof(upf_step_stats, kinetic_energy),'
                   ' sizeof(upf_phase_times), sizeof(upf_launch_config), offsetof(upf_launch_config, measured_ms),'
                   ' offsetof(upf_params, search_cell));return 0;}\n')
    exe = tmp_path / "sz"
    cc = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
    subprocess.run([cc, "-I" + INCLUDE, str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    assert int(out[0]) == C.sizeof(UpfParams)
    assert int(out[1]) == C.sizeof(UpfStepStats)
    assert int(out[2]) == UpfParams.scales.offset
    assert int(out[3]) == UpfStepStats.kinetic_energy.offset
    assert int(out[4]) == C.sizeof(UpfPhaseTimes)
    assert int(out[5]) == C.sizeof(UpfLaunchConfig)
    assert int(out[6]) == UpfLaunchConfig.measured_ms.offset
    assert int(out[7]) == UpfParams.search_cell.offset


def test_abi_version(upf_lib):
    assert upf_lib.lib().upf_abi_version() == 1


def test_invalid_arguments_return_status(upf_lib):
    lib = upf_lib.lib()
    assert lib.upf_default_params(None) == 1
    assert lib.upf_params_derive(None) == 1
    msg = lib.upf_last_error().decode()
    assert "upf_params_derive" in msg
    # bad parameters are rejected before any device work
    p = upf_lib.default_params()
    h = C.c_void_p()
    assert lib.upf_create(C.byref(p), 0, 10, C.byref(h)) == 1  # not derived: block_size 0
    assert "invalid parameters" in lib.upf_last_error().decode()
    assert lib.upf_step(None, 1) == 1


def test_host_params_match_oracle(upf_lib, oracle_lib):
    from unifiedparticleframeworkcuda_b200 import scenes
    for sc in (scenes.small_wcsph(), scenes.small_pcisph(), scenes.wcsph_dam(), scenes.pcisph_dam(8, 8, 8)):
        a = upf_lib.derive_params(sc.params).as_dict()
        b = oracle_lib.derive(sc.params).as_dict()
        da, db = a.pop("density_error_factor"), b.pop("density_error_factor")
        # the neighbour-search cell is the library's own (the lists do not depend on it)
        cell = a.pop("search_cell")
        b.pop("search_cell")
        assert cell >= 4 and cell & (cell - 1) == 0 and cell <= a["block_size"]
        assert a == b
        # FP64 accumulation in the library vs the FP32 restatement
        assert abs(da - db) <= 1e-5 * max(abs(db), 1e-30)


def test_host_luts_bit_equal_to_reference_fixture(upf_lib):
    g = np.load(os.path.join(ROOT, "tests", "golden", "reference_tables.npz"))
    for h, ref in zip(g["lut_h"], g["luts"]):
        p = upf_lib.default_params()
        p.support_radius = float(h)
        got = upf_lib.build_luts(p)
        assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


def test_no_device_means_error_not_fallback(upf_lib):
    """Without a GPU the library refuses to create a system (there is no CPU
    path to fall back to)."""
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("GPU present")
    from unifiedparticleframeworkcuda_b200 import UpfError, scenes
    sc = scenes.small_pcisph()
    with pytest.raises(UpfError) as e:
        upf_lib.ParticleSystem(sc.params, capacity=sc.n)
    assert e.value.status == 9  # UPF_ERR_NO_DEVICE


def test_bin_300_starts_no_later_than_the_support_edge(upf_lib):
    """At these h, (int)(h * (float)(1/h) * 300) is 299, so the first r2 of
    bin 300 would lie above h^2 and a pair just outside the support (which the
    reference skips) would take bin 299; the table starts bin 300 at the
    support's edge instead. Every other h keeps its exact bin-300 threshold.
    (The GPU density-pass bins are checked against the reference rule at
    these h in the GPU parity tests.)"""
    for h in (0.021382991998565044, 0.02923523891741497, 0.05760840918395471):
        p = upf_lib.default_params()
        p.support_radius = h
        thr = upf_lib.bin_thresholds(p)
        hf = np.float32(h)
        factor = np.float32(1.0 / np.float64(hf))
        assert int(np.float32(np.float32(hf * factor) * np.float32(300))) == 299
        assert thr[300] == thr[301]
    rng = np.random.default_rng(5)
    for h in rng.uniform(0.005, 0.2, 200):
        p = upf_lib.default_params()
        p.support_radius = float(h)
        thr = upf_lib.bin_thresholds(p)
        assert thr[300] <= thr[301]


def test_bin_thresholds_reproduce_sqrt_binning(upf_lib):
    """The device derives table bins from r^2 with these thresholds; they must
    give exactly (int)(sqrtf(r2) * (float)(1/h) * 300) and sqrtf(r2) < h."""
    rng = np.random.default_rng(3)
    for h in (0.02, 0.04, 0.0500005, 0.0123):
        p = upf_lib.default_params()
        p.support_radius = h
        thr = upf_lib.bin_thresholds(p)
        hf = np.float32(h)
        factor = np.float32(1.0 / np.float64(hf))
        r2 = np.concatenate([rng.uniform(0, 1.1, 200000).astype(np.float32) * hf * hf,
                             thr[1:].copy(), np.nextafter(thr[1:], np.float32(0))]).astype(np.float32)
        d = np.sqrt(r2, dtype=np.float32)
        exact = ((d * factor).astype(np.float32) * np.float32(300)).astype(np.float32).astype(np.int64)
        got = np.searchsorted(thr[1:301], r2, side="right")  # number of thresholds <= r2
        inside = d < hf
        assert np.array_equal(r2 < thr[301], inside)
        assert np.array_equal(np.minimum(exact, 300)[inside], got[inside])


def test_scratch_for_a_capacity_serves_every_smaller_count(upf_lib):
    """The radix sort's scratch size (host arithmetic): a system allocates it
    for its capacity and sorts any count up to it, so it never shrinks as the
    count grows, across the sizes where the sort's tile changes."""
    f = upf_lib.lib().upf_radix_sort_temp_bytes
    prev = 0
    for n in list(range(0, 5000, 7)) + list(range(262_000, 263_000, 3)) + list(range(1_048_000, 1_049_500, 5)):
        b = f(n)
        assert b >= prev, n
        prev = b


INTEGRATION_CPP = r"""
#include "upf.h"
#include <cstdio>
#include <cstring>
#include <vector>

// the host-side calls the reference's facade makes (InitCudaVariables,
// CudaParticlePhysics, CopyGPUParticles, UnifiedIO), with stand-in data
int main(int argc, char** argv) {
  upf_params p;
  upf_default_params(&p);
  p.method = UPF_METHOD_PCISPH;
  p.particle_spacing = 0.01f;
  p.support_radius = 0.02f;
  p.dt = 5e-4f;
  for (int a = 0; a < 3; ++a) {
    p.container_min[a] = 0.0f;
    p.container_max[a] = 0.3f;
    p.collision_min[a] = 0.005f;
    p.collision_max[a] = 0.295f;
  }
  if (upf_params_derive(&p) != UPF_OK) return 2;
  const uint32_t n = 8;
  std::vector<float> pos(4 * n), vel(4 * n, 0.0f), rho(n), prs(n);
  std::vector<int32_t> type(n, UPF_LIQUID);
  for (uint32_t i = 0; i < n; ++i) {
    pos[4 * i] = 0.1f + 0.01f * (i & 1);
    pos[4 * i + 1] = 0.1f + 0.01f * ((i >> 1) & 1);
    pos[4 * i + 2] = 0.1f + 0.01f * (i >> 2);
  }
  upf_system* s = nullptr;
  upf_status st = upf_create(&p, 0, n, &s);
  if (st == UPF_OK) {
    if (upf_set_particles(s, pos.data(), vel.data(), type.data(), n) != UPF_OK) return 3;
    if (upf_step(s, 1) != UPF_OK) return 4;
    uint32_t got = 0;
    if (upf_get_particles(s, pos.data(), vel.data(), rho.data(), prs.data(), type.data(), nullptr, &got) != UPF_OK)
      return 5;
    upf_destroy(s);
  }
  std::printf("create %d %s\n", (int)st, st == UPF_OK ? "" : upf_last_error());
  // UnifiedIO: write the PCISPH text file, read it back
  if (upf_io_save_fluid_particles_pcisph(argv[1], pos.data(), vel.data(), type.data(), prs.data(), rho.data(), n) !=
      UPF_OK)
    return 6;
  int32_t count = 0, read = 0;
  if (upf_io_read_fluid_particle_num(argv[1], &count) != UPF_OK || count != (int32_t)n) return 7;
  std::vector<float> p3(3 * n), v3(3 * n), cp(n), pd(n);
  std::vector<int32_t> t(n);
  if (upf_io_read_fluid_particles_pcisph(argv[1], p3.data(), v3.data(), t.data(), cp.data(), pd.data(), count,
                                         &read) != UPF_OK || read != count)
    return 8;
  for (uint32_t i = 0; i < n; ++i)
    for (int a = 0; a < 3; ++a)
      if (p3[3 * i + a] != pos[4 * i + a]) return 9;
  std::printf("io ok\n");
  return 0;
}
"""


def test_facade_calls_compile_link_and_run_from_cpp(upf_lib, tmp_path):
    """The calls the reference's facade makes (its C++ change is shown beside
    the call mapping) compile and link from C++ against the library. Run on
    a machine without a GPU, upf_create returns an error with a message
    instead of falling back, and the host-side file calls round-trip a
    PCISPH-format file exactly."""
    import torch

    src = tmp_path / "facade.cpp"
    src.write_text(INTEGRATION_CPP)
    exe = tmp_path / "facade"
    libdir = os.path.join(ROOT, "unifiedparticleframeworkcuda_b200")
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    subprocess.run([cxx, "-O1", "-I" + INCLUDE, str(src), "-o", str(exe), "-L" + libdir, "-lupf",
                    "-Wl,-rpath," + libdir], check=True)
    r = subprocess.run([str(exe), str(tmp_path / "fluid.txt")], capture_output=True, text=True)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    first = r.stdout.splitlines()[0].split(" ", 2)
    if not torch.cuda.is_available():
        assert first[1] != "0" and len(first) == 3 and first[2].strip()
    assert "io ok" in r.stdout
