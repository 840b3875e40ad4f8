"""Generates the golden fixtures in tests/golden/ from the reference's own code.

Host fixtures (run in the container that has the reference checkout; they use
oracle/_ref/libref_host.so, i.e. the reference's Config.cpp, Aggregate.cpp,
OutputWriter.cpp and DiskInit.cpp compiled from their sources):

    python tests/golden/make_golden.py

* fof_*.npz            -- detectAggregates on seeded clustered inputs:
                          per-particle labels / uint16 sizes and the aggregate
                          records (ordered by smallest member)
* writer_run/          -- frames.bin + stats.csv written by OutputWriter for a
                          scripted 3-frame run with aggregates and perturber rows
* config_cases.json    -- loadConfig results / error messages for the config
                          files under tests/golden/configs/
* radius.json          -- particlePhysicalRadius for several masses

GPU fixtures (run on a GPU box; oracle/_ref/libref_engine_nofma.so is the
reference's src/physics/*.cu compiled with -fmad=false):

    python tests/golden/make_golden.py --gpu

* ref_engine_*.npz     -- sort_idx and forces after build/summarize/sort/force,
                          and the state after 3 steps of src/main.cu:101-139
                          (collisions, gas drag, perturber) for seeded disks.
"""
from __future__ import annotations

import argparse
import glob
import importlib
import json
import os
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)

FOF_CASES = [  # (name, seed, n, clusters, spread, link_length)
    ("fof_a", 11, 1200, 30, 0.004, 0.003),
    ("fof_b", 12, 2500, 60, 0.002, 0.0025),
    ("fof_c", 13, 600, 5, 0.05, 0.02),
]


def clustered(seed, n, k, spread):
    rng = np.random.default_rng(seed)
    c = rng.random((k, 3)).astype(np.float32)
    p = c[rng.integers(0, k, n)] + rng.standard_normal((n, 3)).astype(np.float32) * spread
    v = rng.standard_normal((n, 3)).astype(np.float32)
    return [np.ascontiguousarray(a, np.float32) for a in (*p.T, *v.T)]


def host_fixtures():
    import oracle
    ref = oracle.RefHost()
    for name, seed, n, k, spread, ll in FOF_CASES:
        x, y, z, vx, vy, vz = clustered(seed, n, k, spread)
        labels, size, ng, aggs = ref.detect_aggregates(x, y, z, vx, vy, vz, ll, 3.003e-7)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), x=x, y=y, z=z, vx=vx, vy=vy, vz=vz,
                            link_length=np.float32(ll), particle_mass=np.float32(3.003e-7),
                            labels=labels, agg_size=size, n_groups=np.int32(ng),
                            g_n=aggs["n"], g_mass=aggs["mass"], g_c=aggs["c"], g_v=aggs["v"],
                            g_dist=aggs["dist"], g_label=aggs["label"])
        print(name, "groups", ng)

    # scripted writer run
    out = os.path.join(HERE, "writer_run")
    shutil.rmtree(out, ignore_errors=True)
    os.makedirs(out)
    n = 7
    rng = np.random.default_rng(3)
    x, y, z = [np.ascontiguousarray(rng.standard_normal(n) * 3, np.float32) for _ in range(3)]
    agg = np.array([1, 3, 3, 1, 3, 2, 2], np.uint16)
    t = np.array([0.05, 0.1, 0.15000001], np.float32)
    g_n = np.array([3, 2], np.int32)
    g_mass = np.array([3 * 3.003e-7, 2 * 3.003e-7], np.float32)
    g_c = np.array([0.1, -2.5, 1e-3, 4.25, 0.0, -7.125], np.float32)
    g_v = np.array([0.3, 0.001, -0.25, 1.5, 2.5e-5, 0.75], np.float32)
    g_dist = np.array([2.502, 8.2695], np.float32)
    pert = np.array([5.2, 0.0, 0.0, 9.5479e-4, 0.0843, 5.19, 0.0, 0.33, 9.5479e-4, 0.0843,
                     5.17, 0.0, 0.66, 9.5479e-4, 0.0843], np.float32)
    F = oracle._F
    import ctypes as C
    err = C.create_string_buffer(512)
    rc = ref.lib.ref_write_run(out.encode(), n, np.float32(0.005), 10, x.ctypes.data_as(F),
                               y.ctypes.data_as(F), z.ctypes.data_as(F),
                               agg.ctypes.data_as(oracle._U16), 3, t.ctypes.data_as(F), 2,
                               g_n.ctypes.data_as(oracle._I), g_mass.ctypes.data_as(F),
                               g_c.ctypes.data_as(F), g_v.ctypes.data_as(F),
                               g_dist.ctypes.data_as(F), 1, pert.ctypes.data_as(F), err, 512)
    assert rc == 0, err.value
    np.savez(os.path.join(out, "inputs.npz"), x=x, y=y, z=z, agg=agg, t=t, g_n=g_n,
             g_mass=g_mass, g_c=g_c, g_v=g_v, g_dist=g_dist, pert=pert, n=n, dt=np.float32(0.005),
             output_every=10)

    # configs
    cases = {}
    for path in sorted(glob.glob(os.path.join(HERE, "configs", "*.json"))):
        try:
            cases[os.path.basename(path)] = {"ok": True, "cfg": ref.load_config(path)}
        except RuntimeError as e:
            cases[os.path.basename(path)] = {"ok": False, "error": str(e)}
    try:
        ref.load_config(os.path.join(HERE, "configs", "does_not_exist.json"))
    except RuntimeError as e:
        cases["does_not_exist.json"] = {"ok": False, "error": str(e)}
    with open(os.path.join(HERE, "config_cases.json"), "w") as f:
        json.dump(cases, f, indent=1, sort_keys=True)

    masses = [3.003e-7, 3.003e-6, 1e-8, 1e-9, 2.5e-5]
    with open(os.path.join(HERE, "radius.json"), "w") as f:
        json.dump({repr(m): float(ref.particle_radius(m)) for m in masses}, f, indent=1)


def gpu_fixtures():
    import oracle
    nb = importlib.import_module("nbody-sim_b200")
    port = oracle.Port()
    for seed, n in ((21, 1024), (22, 3000)):
        d = nb.make_disk(n, 0.5, 5.0, 0.01, 0.005, 1.0, seed)
        st = {k: v.astype(np.float32) for k, v in d.items()}
        st["m"] = np.full(n, 1e-8, np.float32)
        t = port.build_tree(st["x"], st["y"], st["z"], st["m"])
        info = port.tree_info(t)
        port.free_tree(t)
        assert info.lost_bodies == 0 and info.unsummarized == 0 and info.height <= 20
        eng = oracle.RefEngine(n, nofma=True)
        eng.set_state(st)
        si, root_mass, root_count, next_node = eng.build()
        eng.force(0.5, 1e-3, 1.0)
        f = eng.get_state()
        # 3 steps with collisions (factor 500), drag and a perturber
        r_coll = np.float32(500.0) * np.float32(nb.particle_physical_radius(1e-8))
        pert = port.perturber(True, 1.0, 5.2, 0.0, 1.0)
        eng.force(0.5, 1e-3, 1.0, pert=pert)
        eng.steps(0, 3, 0.01, 0.5, 1e-3, 1.0, float(r_coll), 0.0, 1e-2, True, 1.0, 5.2, 0.0)
        s3 = eng.get_state()
        eng.close()
        np.savez_compressed(os.path.join(HERE, f"ref_engine_{n}.npz"), **{k: st[k] for k in st},
                            sort_idx=si, root_count=np.int32(root_count),
                            ax=f["ax"], ay=f["ay"], az=f["az"],
                            **{"s3_" + k: s3[k] for k in s3}, r_coll=r_coll)
        print("ref engine fixture", n)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpu", action="store_true")
    a = ap.parse_args()
    if a.gpu:
        gpu_fixtures()
    else:
        host_fixtures()
