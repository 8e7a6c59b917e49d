"""One forward 3x3 convolution of the warm-start network, as a target for
ncu captures.

    python -m musoc_solver_b200.profile_conv --H 600 --W 904 --cin 256 --cout 256 --path tma

Random BF16 activations [H*W][cin] and K-major weights [9][cout][cin]; runs
the chosen tcgen05 kernel (``tma``: tensor-map loads; ``tc``: cp.async
loads) `--reps` times and checks the timeout flag.
"""
from __future__ import annotations

import argparse
import ctypes as C


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--H", type=int, default=600)
    ap.add_argument("--W", type=int, default=904)
    ap.add_argument("--cin", type=int, default=256)
    ap.add_argument("--cout", type=int, default=256)
    ap.add_argument("--path", choices=["tma", "tc"], default="tma")
    ap.add_argument("--reps", type=int, default=3)
    args = ap.parse_args(argv)
    import torch

    from . import build
    from .unet import lib

    build.build()
    L = lib()
    g = torch.Generator(device="cuda").manual_seed(0)
    P = args.H * args.W
    x = torch.randn(P, args.cin, device="cuda", generator=g).to(torch.bfloat16)
    wk = (torch.randn(9, args.cout, args.cin, device="cuda", generator=g) / 30).to(torch.bfloat16)
    b = torch.zeros(args.cout, device="cuda")
    y = torch.zeros(P, args.cout, dtype=torch.bfloat16, device="cuda")
    fn = L.sevp_nn_conv3x3_tma if args.path == "tma" else L.sevp_nn_conv3x3_tc
    p = lambda t: C.c_void_p(t.data_ptr())
    for _ in range(args.reps):
        s = fn(p(x), args.cin, 0, args.cin, p(wk), p(b), p(y), args.cout, 0, args.cout, 1, args.H,
               args.W, 1, None)
        assert s == 0, s
    code = C.c_int(-1)
    assert L.sevp_nn_tc_status(C.byref(code)) == 0 and code.value == 0
    torch.cuda.synchronize()
    print("ok", args)


if __name__ == "__main__":
    main()
