"""bench.py's added targets (no GPU needed): run_targets turns the results of
its workloads (sparse grid, config 3 forward + adjoint, config 4 and config 5
batched runs) into the keys of the one bench line.  The workload functions
are replaced by stand-ins that return results of the same shape, so this
checks the line's assembly, not the measurements."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_targets_keys_of_the_bench_line(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    import torch

    adj = {"ratio_vs_plain_forward": 2.93, "grad_check": {"direction": "d", "fd": 1.0, "adjoint": 1.0, "rel_err": 4e-6},
           "config": {"n_particles": 262144, "timing": "median of 3"}, "steps": 256, "plain_forward_ms": 13.9,
           "forward_adjoint_ms": 40.7, "value": 1.6e9,
           "replays": {"sort_record": True, "replayed_steps_sorted_again": 0}}

    def batched(args, device, adjoint, steps):
        return {"speedup_vs_loop": 1.56 if adjoint else 5.7, "config": {"n_particles": 100}, "steps": steps,
                "batched_ms": 1.0, "loop_ms": 2.0, "value": 1.0, "loop_of_single_scene_value": 0.5}

    monkeypatch.setattr(bench, "run_sparse", lambda args, device: {"ratio": 1.06})
    monkeypatch.setattr(bench, "run_adjoint", lambda args, device: adj)
    monkeypatch.setattr(bench, "run_batched", batched)
    monkeypatch.setattr(torch.cuda, "empty_cache", lambda: None)
    line = bench.run_targets(None, 0)
    assert line["adjoint_ratio_vs_plain"] == 2.93
    assert line["grad_fd_rel_err"] == 4e-6
    assert line["batched_speedup_vs_loop"] == 5.7 and line["batched_adjoint_speedup_vs_loop"] == 1.56
    assert line["sparse_vs_dense_step_ratio"] == 1.06
    cube = line["targets"]["differentiable_elastic_cube"]
    assert cube["target_ratio"] == 3.0 and cube["steps"] == 256 and cube["checkpoint_every"] == 16
    assert cube["replays"] == {"sort_record": True, "replayed_steps_sorted_again": 0}
    assert set(line["targets"]) >= {"sparse_grid_two_material_drop", "differentiable_elastic_cube",
                                    "batched_forward_64_scenes", "batched_forward_adjoint_32_scenes"}
