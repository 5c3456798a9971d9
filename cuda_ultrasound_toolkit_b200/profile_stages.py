"""Runs each pipeline stage once on a synthetic frame, for profilers.

    python -m cuda_ultrasound_toolkit_b200.profile_stages [--workload full] [--repeat 1]
    python -m cuda_ultrasound_toolkit_b200.profile_stages --sequence tpw_fine [--repeat 1]

Launch order: one warm-up pass of decode, Hilbert, delay-and-sum (3 kernels), then `repeat`
passes of the same three kernels. With ncu, skip the warm-up with `-s 3`. With --sequence, the
delay-and-sum of that benchmark sequence workload (synth.sequence_params) on a random analytic
signal resident on the GPU: one warm-up launch, then `repeat` launches (ncu: `-s 1`).
"""
import argparse

import torch

from . import Plan, synth


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="full", choices=sorted(synth.CONFIGS))
    ap.add_argument("--repeat", type=int, default=1)
    ap.add_argument("--bf16", action="store_true", help="store the analytic signal as bf16")
    ap.add_argument("--decode-tc", action="store_true", help="decode on int8 tensor cores")
    ap.add_argument("--schedule", type=int, default=0,
                    help="delay-and-sum schedule: 0 automatic, 1 one CTA per tile, 2 stream-K")
    ap.add_argument("--sequence", default=None, choices=["tpw", "uforces", "tpw_fine", "uforces_fine"],
                    help="profile the delay-and-sum of a TPW / UFORCES workload instead")
    args = ap.parse_args()
    if args.sequence:
        bp = synth.sequence_params(args.sequence)
        plan = Plan(bp, iq_bf16=args.bf16, das_schedule=args.schedule)
        S, C, T = bp.dims
        g = torch.Generator(device="cuda").manual_seed(11)
        iq = torch.complex(torch.randn(T, C, S, device="cuda", generator=g), torch.randn(T, C, S, device="cuda", generator=g))
        vol = plan.empty_volume()
        for _ in range(1 + args.repeat):
            plan.das(iq, out=vol)
        plan.check()
        torch.cuda.synchronize()
        print(f"ok: {args.sequence}, {1 + args.repeat} delay-and-sum launches")
        return
    raw, bp = synth.frame(args.workload)
    plan = Plan(bp, iq_bf16=args.bf16, decode_tc=args.decode_tc, das_schedule=args.schedule)
    d_raw = torch.from_numpy(raw).cuda()
    vol, dec, iq = plan.empty_volume(), plan.empty_decoded(), plan.empty_iq()
    plan.beamform(d_raw, out=vol)
    for _ in range(args.repeat):
        plan.decode(d_raw, out=dec)
        plan.hilbert(dec, out=iq)
        plan.das(iq, out=vol)
    plan.check()
    torch.cuda.synchronize()
    print(f"ok: {args.workload}, {3 * (args.repeat + 1)} kernels")


if __name__ == "__main__":
    main()
