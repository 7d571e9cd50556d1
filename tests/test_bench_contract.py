"""The reference arm of bench.py (the oracle's filter timed on the host cores)
prints one JSON line with the keys the benchmark contract asks for; it runs
on CPU, so it is checked here with a one-step sample."""
import json
import os
import subprocess
import sys

from conftest import ROOT


def test_reference_arm_prints_contract_line():
    env = dict(os.environ)
    env.pop("RANK", None)
    env.pop("WORLD_SIZE", None)
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--steps", "1", "--warmup", "0"], capture_output=True, text=True,
                         timeout=600, cwd=ROOT, env=env)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "scaling", "vs_baseline", "dtype", "config", "cpu_baseline",
              "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0 and d["steps"] == 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert d["e2e"]["value"] == d["value"] and d["cpu_baseline"]["value"] == d["value"]
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert "workload" in d["config"]
    # both arms describe the same workload with the same config dict
    assert d["config"]["n_bands"] == 160 and d["config"]["ndeg"] == 16


def test_reference_arm_loads_no_cuda_library():
    """The reference arm builds its inputs with the oracle's copy of the
    seeded generator: only oracle/ libraries are mapped, never the CUDA
    library of the product."""
    code = ("import sys; sys.path.insert(0, %r); import bench; "
            "t, c, smp, s = bench.reference_steps(1, 0); "
            "maps = open('/proc/self/maps').read(); "
            "print('CUDA_LIB' if 'libchfsi_b200' in maps else 'NO_CUDA_LIB', "
            "'ORACLE' if 'liboracle' in maps else 'NO_ORACLE')" % ROOT)
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                         timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    assert "NO_CUDA_LIB ORACLE" in out.stdout


def test_oracle_generator_is_bit_identical_to_the_library_one():
    import numpy as np
    import chfsi
    import synth
    for cfg in (0, 1):
        a = synth.System(config_index=cfg)
        b = chfsi.SyntheticSystem(config_index=cfg)
        for f in ("miller", "kinetic", "vloc_g", "beta", "proj_offsets", "dmat", "psi0",
                  "occupations", "positions"):
            assert np.array_equal(getattr(a, f)(), getattr(b, f)()), (cfg, f)
