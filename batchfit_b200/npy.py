"""Fit spectra straight from .npy files on the GPU (out of core).

Mirrors the reference's ``batchfit_fit_npy`` tool (tools/fit_npy.cpp:20-121):

    python -m batchfit_b200.npy --x x.npy --y y.npy [--initial initial.npy] --output NEW_DIR \\
        [--model gaussian|lorentzian|pseudo_voigt|two_lorentzian] [--chunk-fits 0] [--in-flight 3] \\
        [--uncertainties] [--policy parity|reference]

y[N,M] is streamed in chunks (never loaded whole); NEW_DIR receives
parameters.npy, chi_squared.npy, status.npy and iterations.npy (plus the
uncertainty outputs with --uncertainties), and the tool prints a one-line summary.
"""

from __future__ import annotations

import argparse
import ctypes as C
import os
import sys

from . import _capi


def fit_npy(x, y, output, model="gaussian", initial=None, bounds=None, *, uncertainties=False, chunk_fits=0,
            in_flight=3, policy="parity", device=0) -> dict:
    """Fit every row of the .npy file ``y`` against the .npy grid ``x``; results are
    written as .npy files into the new directory ``output``.  Returns the run's
    statistics (fits, chunks, chunk_fits and seconds spent reading, fitting,
    writing and in total)."""
    from . import MODELS, _PARAMETERS, _bounds, context, solver_options

    if model not in MODELS:
        raise ValueError(f"unknown model {model!r}; choose one of {tuple(MODELS)}")
    if not 1 <= int(in_flight) <= 3:
        raise ValueError("in_flight must be 1..3")
    lower, upper = _bounds(bounds, _PARAMETERS[model])
    opts = _capi.NpyOptions(MODELS[model], int(bool(uncertainties)), int(chunk_fits), int(in_flight),
                            solver_options(model, lower, upper, policy))
    stats = _capi.NpyStats()
    lib = _capi.load()
    enc = lambda p: None if p is None else os.fsencode(p)  # noqa: E731
    _capi.check(lib.bf_cuda_fit_npy(context(device).handle, enc(x), enc(y), enc(initial), enc(output),
                                    C.byref(opts), C.byref(stats)), "bf_cuda_fit_npy")
    return {name: getattr(stats, name) for name, _ in stats._fields_}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--x", required=True)
    ap.add_argument("--y", required=True)
    ap.add_argument("--initial")
    ap.add_argument("--output", required=True)
    ap.add_argument("--model", default="gaussian")
    ap.add_argument("--chunk-fits", type=int, default=0)
    ap.add_argument("--in-flight", type=int, default=3)
    ap.add_argument("--uncertainties", action="store_true")
    ap.add_argument("--policy", default="parity", choices=("parity", "reference"))
    args = ap.parse_args(argv)
    try:
        s = fit_npy(args.x, args.y, args.output, args.model, args.initial, uncertainties=args.uncertainties,
                    chunk_fits=args.chunk_fits, in_flight=args.in_flight, policy=args.policy)
    except (ValueError, RuntimeError) as error:
        print(error, file=sys.stderr)
        return 1
    print(f"fits={s['fits']} chunks={s['chunks']} chunk_fits={s['chunk_fits']} "
          f"read_seconds={s['read_seconds']:.4f} fit_seconds={s['fit_seconds']:.4f} "
          f"write_seconds={s['write_seconds']:.4f} wall_seconds={s['wall_seconds']:.4f} "
          f"fits_per_second={s['fits'] / max(s['wall_seconds'], 1e-12):.1f}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
