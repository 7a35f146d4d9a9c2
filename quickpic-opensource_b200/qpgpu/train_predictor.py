"""Train the learned start of the B predictor-corrector passes on the GPU.

The training pairs come from the plain solver itself: simulations drawn over
the parameter-scan ranges run one 3D step each with the B passes iterated to a
relative change of 1e-4 from the carried start (the reference's), and every
slice records one pair (Simulation.record).  The network is then trained with
the engine's own tensor-core kernels (Predictor.train) and evaluated on
held-out simulations: passes per slice from the carried start, the quadratic
extrapolation and the learned start, at the same tolerance.

Ranges (the batched parameter scan's): transverse grids 128^2, 256^2, 512^2
drawn log-uniform, 2 x 2 particles per cell, tri-Gaussian beam with nb/np
log-uniform in [0.5, 20] and sigma_r uniform in [0.1, 0.5] c/wp (a pair with
(nb/np) sigma_r^2 > 1, a full blow-out, is drawn again), beam particles in
proportion to the grid area (262,144 at 128^2, at most 2,097,152), gamma =
20000, over a 12 x 12 x 10 c/wp box.  The scan's 256 slices and sigma_z = 0.5
c/wp are widened to 256 or 512 slices and sigma_z uniform in [0.4, 0.7] c/wp,
so that the slice width (a feature of the network) and the bunch length of the
512-slice medium case are inside the training set.

    python quickpic-opensource_b200/qpgpu/train_predictor.py --pairs 20000 \
        --out quickpic-opensource_b200/qpgpu/predictor_weights.npy
"""
import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
if os.path.dirname(HERE) not in sys.path:
    sys.path.insert(0, os.path.dirname(HERE))

import qpgpu  # noqa: E402

BOX = [[-6.0, 6.0], [-6.0, 6.0], [0.0, 10.0]]


def draw_instances(n, seed):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        ind = int(rng.integers(7, 10))
        while True:
            peak = float(np.exp(rng.uniform(np.log(0.5), np.log(20.0))))
            sr = float(rng.uniform(0.1, 0.5))
            if peak * sr * sr <= 1.0:
                break
        nb = {7: [64, 64, 64], 8: [128, 128, 64], 9: [128, 128, 128]}[ind]
        nz_ind = int(rng.integers(8, 10))
        sz = float(rng.uniform(0.4, 0.7))
        out.append(dict(ind=ind, peak=peak, sigma_r=sr, sigma_z=sz, nz_ind=nz_ind, np=nb))
    return out


def make_sim(inst, predict=0, tol=1e-4, iter=16, device=0):
    c = qpgpu.Context(inst["ind"], inst["ind"], inst["nz_ind"], BOX, device=device)
    sp = qpgpu.Species2d(c, ppc=(2, 2))
    bm = qpgpu.Beam3d(c, inst["np"], q=-1.0, m=1.0, gamma=20000.0, peak_density=inst["peak"],
                      quiet_start=True, center=[0.0, 0.0, 2.5],
                      sigma=[inst["sigma_r"], inst["sigma_r"], inst["sigma_z"]],
                      sigma_v=[0.0, 0.0, 0.0])
    sim = qpgpu.Simulation(c, [sp], [bm], iter=iter, store3d=False, tol=tol, predict=predict)
    return c, sp, bm, sim


def close(*objs):
    for o in objs:
        o.close()


def record(data, instances, device=0):
    """Record one step of each instance.  An instance whose plasma electrons
    leave the grid (a strong blow-out can send an electron across the box in
    one slice; the engine stops the step with an error, as the reference's
    push has no guard for it either) keeps the pairs of the slices before."""
    failed = 0
    for inst in instances:
        if len(data) >= data.capacity:
            break
        c, sp, bm, sim = make_sim(inst, device=device)
        sim.record(data)
        try:
            sim.step3d()
        except qpgpu.QPError:
            failed += 1
        close(sim, bm, sp, c)
    return failed


def evaluate(net, instances, device=0):
    """Passes per slice from the carried (0), quadratic (2) and learned (3) starts."""
    tot = {0: 0, 2: 0, 3: 0}
    slices = 0
    for inst in instances:
        got = {}
        for predict in (0, 2, 3):
            c, sp, bm, sim = make_sim(inst, predict=predict, device=device)
            if predict == 3:
                sim.set_predictor(net)
            try:
                got[predict] = sim.step3d()
            except qpgpu.QPError:
                pass
            close(sim, bm, sp, c)
        if len(got) == 3:  # instances that ran in every mode
            for k, st in got.items():
                tot[k] += st.iterations
            slices += got[0].slices
    return {k: v / max(slices, 1) for k, v in tot.items()}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--pairs", type=int, default=20000)
    ap.add_argument("--steps", type=int, default=6000)
    ap.add_argument("--batch", type=int, default=32)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--eval", type=int, default=6, help="held-out simulations")
    ap.add_argument("--out", default=os.path.join(HERE, "predictor_weights.npy"))
    args = ap.parse_args()
    per = 384  # slices per instance, on average
    n_inst = (args.pairs + per - 1) // per
    t0 = time.time()
    data = qpgpu.TrainingSet(args.pairs)
    failed = record(data, draw_instances(n_inst + 8, args.seed))
    t_rec = time.time() - t0
    net = qpgpu.Predictor(seed=args.seed)
    st = net.train(data, steps=args.steps, batch=args.batch, lr=args.lr, seed=args.seed + 1)
    held = draw_instances(args.eval, args.seed + 7919)
    ev = evaluate(net, held)
    np.save(args.out, net.get_params())
    info = {"pairs": len(data), "instances": n_inst, "instances_stopped": failed,
            "record_s": round(t_rec, 1),
            "steps": args.steps, "batch": args.batch, "lr": args.lr,
            "first_loss": st.first_loss, "last_loss": st.last_loss,
            "train_gpu_ms": st.gpu_ms,
            "held_out_passes_per_slice": {"carried": ev[0], "quadratic": ev[2], "learned": ev[3]},
            "held_out": args.eval, "seed": args.seed}
    with open(os.path.splitext(args.out)[0] + ".json", "w") as f:
        json.dump(info, f, indent=1)
    print(json.dumps(info), flush=True)
    close(net, data)


if __name__ == "__main__":
    main()
