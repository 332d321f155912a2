"""Operator timing on a 3-D koosh-ball case of chosen size: builds Gu/Gut and
a NUFFT plan, runs `reps` forward (Shanna) and adjoint (Nakatsha) operator
applications, and prints the per-stage CUDA-event times of the plan's
stage profiler (forward x/y/z line-FFT passes, Gu, Gut, inverse z/y/x).

A small case keeps profiler captures short, e.g.

    python -m monalisa_b200.opbench --n 64 --spokes 1024 --samples 128 --coils 16

(64^3 image, 128^3 grid: the grid, 268 MB, and the pass buffers still exceed
the 126 MB L2).  The headline workload is --n 128 --spokes 4096 --samples 256.
"""
import argparse

import numpy as np

STAGES = ["fwd_x", "fwd_y", "fwd_z", "gu", "gut", "inv_z", "inv_y", "inv_x"]


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--n", type=int, default=64, help="image edge (grid edge 2n)")
    ap.add_argument("--spokes", type=int, default=1024)
    ap.add_argument("--samples", type=int, default=128, help="samples per spoke")
    ap.add_argument("--coils", type=int, default=16)
    ap.add_argument("--reps", type=int, default=3, help="forward + adjoint applications")
    ap.add_argument("--adjoint", default="masked", choices=["masked", "fused", "full_grid"])
    ap.add_argument("--precision", default="fp32", choices=["fp32", "mixed", "fp16_values"])
    ap.add_argument("--buffers", type=int, default=None, choices=[0, 2, 3],
                    help="line-FFT passes: TMA with 2 or 3 bundle buffers, or 0 (cp.async); default: the plan's")
    ap.add_argument("--masked-store", type=int, default=None, choices=[0, 1],
                    help="last forward pass stores only grid chunks Gu reads (1) or the whole grid (0)")
    ap.add_argument("--records", type=int, default=None, choices=[0, 1],
                    help="Gut rows from row records (1) or the CSR (0); default: the plan's")
    ap.add_argument("--op", default="nufft", choices=["nufft", "gridder"],
                    help="nufft: operator stages; gridder: the leight adjoint gridder on the samples")
    args = ap.parse_args(argv)

    import torch

    import monalisa_b200 as mb
    from monalisa_b200 import _native as N
    from monalisa_b200 import traj

    n, Ng = args.n, 2 * args.n
    t = traj.bmTraj_fullRadial3_phyllotaxis_lineAssym2(args.samples, args.spokes, 1, Ng / args.samples)
    ve = traj.bmVolumeElement_full_radial3(t)
    if args.op == "gridder":
        rng = np.random.default_rng(7)
        data = (rng.standard_normal((args.coils, t.shape[1])) +
                1j * rng.standard_normal((args.coils, t.shape[1]))).astype(np.complex64)
        for _ in range(max(1, args.reps)):
            mb.gridding.bmGridder_n2u_leight_dev(data, t, ve, [Ng] * 3, [1, 1, 1], "gauss", 3, [0.61, 10])
        torch.cuda.synchronize()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        ev[0].record()
        mb.gridding.bmGridder_n2u_leight_dev(data, t, ve, [Ng] * 3, [1, 1, 1], "gauss", 3, [0.61, 10])
        ev[1].record()
        torch.cuda.synchronize()
        print(f"leight gridder {t.shape[1]} samples, {args.coils} coils -> {Ng}^3: "
              f"{ev[0].elapsed_time(ev[1]):.3f} ms (with host preparation and upload)")
        return
    Gu, Gut = mb.bmTraj2SparseMat(t, ve, [Ng] * 3, [1, 1, 1])
    rec = mb.SensaRecon(Gu, Gut, traj.coil_maps([n] * 3, args.coils, 1), [n] * 3, precision=args.precision)
    rec.plan.adjoint_mode = args.adjoint
    if args.buffers is not None:
        rec.plan.variant = {"pass_buffers": args.buffers}
    if args.records is not None:
        rec.plan.variant = {"gut_records": args.records}
    if args.masked_store is not None:
        rec.plan.variant = {"fwd_masked_store": args.masked_store}
    x = torch.from_numpy(traj.ellipsoid_phantom([n] * 3, 5, 2)).cuda()
    for _ in range(args.reps):
        y = rec.plan.shanna(x)
        rec.plan.nakatsha(y)
    torch.cuda.synchronize()
    ms = np.zeros(len(STAGES))
    N.call("mlg_plan_profile", rec.plan.handle, max(1, args.reps), N.dptr(ms))
    print(f"{n}^3 image, {Ng}^3 grid, {args.spokes}x{args.samples} samples, {args.coils} coils, "
          f"adjoint {rec.plan.adjoint_mode}, precision {args.precision}, variant {rec.plan.variant}, "
          f"fp16 intermediate {rec.plan.half_intermediate and args.precision == 'mixed'}, Gu nnz {Gu.nnz}")
    for name, v in zip(STAGES, ms):
        print(f"  {name:6s} {v:8.4f} ms")
    rec.plan.close()


if __name__ == "__main__":
    main()
