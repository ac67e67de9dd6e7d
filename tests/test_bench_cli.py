"""bench.py's reference arm (the reference's own program compiled for the
host, with the oracle port beside it) runs without a GPU: check its JSON
line on a short run, and that ranks other than 0 of a multi-rank launch
exit quietly."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run(args, env=None):
    e = dict(os.environ)
    e.update(env or {})
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py")] + args,
                          capture_output=True, text=True, cwd=ROOT, env=e, timeout=600)


def test_reference_arm_line():
    p = run(["--impl", "reference", "--steps", "2", "--warmup", "3", "--cpu-rays", "64"])
    assert p.returncode == 0, p.stderr[-2000:]
    line = json.loads(p.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["metric"] == "ray-steps/s"
    assert line["value"] > 0 and line["higher_is_better"] is True
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    base = line["cpu_baseline"]
    assert base["cores"] >= 1
    if O.ref_available():  # the reference's own program, the restatement beside it
        assert base["kind"] == "reference" and base["port"]["kind"] == "port"
        assert base["port"]["value"] > 0
    else:
        assert base["kind"] == "port"
    assert line["e2e"] == {"value": line["value"], "unit": "ray-steps/s",
                           "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert line["config"]["workload"] == "torus_rt_1024"


def test_reference_arm_numerical_is_unavailable():
    """numerical_128's grid is generated on the GPU, so the reference arm
    says so on one line and exits 0 instead of timing the wrong program."""
    p = run(["--impl", "reference", "--workload", "numerical_128", "--steps", "1", "--warmup", "3"])
    assert p.returncode == 0, p.stderr[-2000:]
    line = json.loads(p.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and "unavailable" in line


def test_reference_arm_other_ranks_exit_quietly():
    p = run(["--impl", "reference", "--steps", "1", "--warmup", "3", "--gpus", "2"],
            env={"RANK": "1", "LOCAL_RANK": "1", "WORLD_SIZE": "2"})
    assert p.returncode == 0, p.stderr[-2000:]
    assert p.stdout.strip() == ""


def test_cpu_legs_time_one_fixed_sample():
    """The GPU arm's cpu_baseline leg and the reference arm time the same
    fixed ray sample (the same indices, every dump interval) split the same
    way, with the same programs (the restatement, and the reference's own
    program where it was built), so their rates differ only by timing noise;
    the FP32 build of the restatement is reported beside the FP64 one with
    its image error."""
    import argparse
    import sys
    sys.path.insert(0, ROOT)
    import bench
    from gray_b200 import configs
    cfg = configs.scaled(configs.TORUS_RT_1024, 32)
    rays = bench.cpu_sample(32 * 32, 64)
    assert len(set(rays.tolist())) == 64 and rays.max() < 32 * 32
    assert list(rays) == list(bench.cpu_sample(32 * 32, 64))  # fixed: the same every run
    args = argparse.Namespace(cpu_rays=64, steps=3, workload="torus_rt_1024")
    res = bench.analytic_cpu(cfg, args)
    assert res["kind"] == "port" and res["precision"] == "fp64" and res["value"] > 0
    assert "64 rays" in res["sample"] and "in 3 parts" in res["sample"]
    assert res["fp32"]["value"] > 0 and res["fp32"]["image_rel_l2_err_vs_fp64"] > 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    if O.ref_available():
        assert res["reference_program"]["kind"] == "reference"
        assert res["reference_program"]["value"] > 0
    p = run(["--impl", "reference", "--steps", "3", "--warmup", "3", "--cpu-rays", "64",
             "--side", "32"])
    assert p.returncode == 0, p.stderr[-2000:]
    line = json.loads(p.stdout.strip().splitlines()[-1])
    assert "64 rays" in line["cpu_baseline"]["sample"] and "in 3 parts" in line["cpu_baseline"]["sample"]
