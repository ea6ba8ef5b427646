"""Failure detection without a GPU fault: every failure is made on the host
(bad input, an injected allocation failure, a too-small capacity) or is a
bounded device wait that is allowed to run out; each must come back as a
status code with the context still usable."""
import numpy as np
import pytest

from unifiedparticleframeworkcuda_b200 import STATUS, UpfError, scenes

pytestmark = pytest.mark.gpu

CODE = {name: code for code, name in STATUS.items()}


def status_of(exc):
    return exc.value.status


def small_system(upf, sc, **over):
    p = upf.derive_params(sc.params)
    for k, v in over.items():
        setattr(p, k, v)
    s = upf.ParticleSystem(p, capacity=sc.n, derive=False)
    return s


def test_nan_input_is_reported_not_propagated(upf_lib):
    sc = scenes.small_pcisph()
    pos = sc.pos.copy()
    k = int(np.flatnonzero(sc.type == 2)[5])
    pos[k, 1] = np.nan
    with small_system(upf_lib, sc) as s:
        s.set_particles(pos, sc.vel, sc.type)
        s.step(1)
        with pytest.raises(UpfError) as e:
            s.synchronize()
        assert status_of(e) == CODE["UPF_ERR_NAN"]
    # the device is fine afterwards
    with small_system(upf_lib, sc) as s:
        s.set_particles(sc.pos, sc.vel, sc.type)
        s.step(2)
        s.synchronize()


def test_neighbor_overflow_is_reported(upf_lib):
    sc = scenes.small_pcisph()
    with small_system(upf_lib, sc, max_neighbors=8) as s:
        s.set_particles(sc.pos, sc.vel, sc.type)
        s.step(1)
        with pytest.raises(UpfError) as e:
            s.synchronize()
        assert status_of(e) == CODE["UPF_ERR_NEIGHBOR_OVERFLOW"]
        assert "max_neighbors=8" in str(e.value)


def test_bounded_wait_runs_out_and_the_context_survives(upf_lib):
    L = upf_lib.lib()
    rc = L.upf_selftest_bounded_wait(0, 2000)  # 2 ms
    assert rc == CODE["UPF_ERR_TIMEOUT"]
    assert "bounded" in L.upf_last_error().decode()
    sc = scenes.small_pcisph()
    with small_system(upf_lib, sc) as s:
        s.set_particles(sc.pos, sc.vel, sc.type)
        s.step(2)
        s.synchronize()


def test_injected_allocation_failures(upf_lib):
    L = upf_lib.lib()
    sc = scenes.small_pcisph()
    p = upf_lib.derive_params(sc.params)
    try:
        for nth in (0, 5, 20):
            L.upf_test_fail_allocation(nth)
            with pytest.raises(UpfError) as e:
                upf_lib.ParticleSystem(p, capacity=sc.n, derive=False)
            assert status_of(e) == CODE["UPF_ERR_ALLOC"] and "injected" in str(e.value)
        scs = scenes.batch_scenes(num=2, seed=3, counts=(2048, 4096))
        L.upf_test_fail_allocation(7)
        with pytest.raises(UpfError) as e:
            upf_lib.ParticleBatch([x.params for x in scs], [x.n for x in scs])
        assert status_of(e) == CODE["UPF_ERR_ALLOC"]
        a = scenes.adjoint_scene(8, 8, 8)
        L.upf_test_fail_allocation(3)
        with pytest.raises(UpfError) as e:
            upf_lib.Adjoint(a.params, a.pos, a.vel, steps=4)
        assert status_of(e) == CODE["UPF_ERR_ALLOC"]
    finally:
        L.upf_test_fail_allocation(-1)
    # everything allocated before each failure was released: a full system works
    with upf_lib.ParticleSystem(p, capacity=sc.n, derive=False) as s:
        s.set_particles(sc.pos, sc.vel, sc.type)
        s.step(1)
        s.synchronize()
