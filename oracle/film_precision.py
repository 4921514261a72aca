"""What the FP64 film changes against the reference's FP32 Kahan film.

    python -m oracle.film_precision [--size 512] [--spp 4096] [--threads 0]

Renders the Cornell box (max path length 8) once with the CPU restatement of
path_tracing.cu and feeds every sample's contribution to three films at
once: FP64 (as the CUDA renderers accumulate), the reference's own FP32
SpectrumStorage (Kahan pairs per stratum, spectrum_types.h:662-697) and a
plain FP32 sum.  Prints, as one JSON line, the relative difference of the
FP32 films from the FP64 film per stratum and per pixel (CIE Y), max and
mean over the pixels.  TEST INFRASTRUCTURE: runs on the host only.
"""
import argparse
import json
import time

import numpy as np

from oracle import ref


def measure(size=512, spp=4096, threads=0):
    from vlr_b200 import scenes
    desc = scenes.cornell_box_desc(size, size)
    t0 = time.time()
    f64, kahan, plain, _ = ref.pt_render_fp32_films(scenes.flatten_desc(desc), desc["camera"], size, size, spp, 8,
                                                    threads=threads)
    seconds = time.time() - t0
    _, _, cmf, _ = ref.tables()
    ybar = cmf[1].astype(np.float64)

    def rel(a):
        a = a.astype(np.float64)
        lit = f64 > 0
        per_stratum = np.abs(a - f64)[lit] / f64[lit]
        y64, y32 = f64 @ ybar, a @ ybar
        ylit = y64 > 1e-6 * y64.max()
        per_pixel = np.abs(y32 - y64)[ylit] / y64[ylit]
        return {"stratum_max": float(per_stratum.max()), "stratum_mean": float(per_stratum.mean()),
                "pixel_y_max": float(per_pixel.max()), "pixel_y_mean": float(per_pixel.mean()),
                "image_y_rel": float(abs(y32.sum() / y64.sum() - 1))}

    return {"scene": "Cornell box", "size": size, "spp": spp, "seconds": seconds,
            "fp32_kahan_vs_fp64": rel(kahan), "fp32_plain_vs_fp64": rel(plain)}


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--size", type=int, default=512)
    ap.add_argument("--spp", type=int, default=4096)
    ap.add_argument("--threads", type=int, default=0)
    a = ap.parse_args()
    print(json.dumps(measure(a.size, a.spp, a.threads)))
