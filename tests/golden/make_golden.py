"""Regenerates the golden fixtures of this directory from the reference's own
code built for the host (oracle/_ref, built by oracle/build_ref.sh from the
reference sources):

  bsdf_batch_2048.npz   2048 seeded BSDF-batch queries and the outputs of the
                        reference's BSDF classes (materials.cu) for them;
  upsample.npz          packed Meng-Simon spectra (spectrum_types.cpp:162-228)
                        of 256 seeded colours per colour space, in every
                        spectrum type;
  pt_cornell_32.npz     CIE Y of the 32x32 Cornell box, 256 spp, max path
                        length 8, from the CPU restatement of path_tracing.cu
                        over the reference's BSDF/spectral classes.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def main():
    import vlr_b200 as V
    from vlr_b200 import scenes
    from oracle import ref
    if not ref.available():
        raise SystemExit("oracle/_ref is not built (run oracle/build_ref.sh)")
    inp = V.make_bsdf_batch_inputs(2048, seed=2024)
    out = ref.bsdf_batch(inp)
    np.savez_compressed(os.path.join(HERE, "bsdf_batch_2048.npz"), **{"in_" + k: v for k, v in inp.items()},
                        **{"out_" + k: v for k, v in out.items()})

    # colour spaces 0 sRGB gamma, 1 Rec.709 linear: RGB in [0, 1.2]; 2 XYZ and
    # 3 xyY: colours of the Rec.709 gamut (chromaticities outside the
    # tabulated gamut are undefined in the reference)
    rng = np.random.default_rng(77)
    rgb = rng.uniform(0, 1.2, (256, 3))
    inner = rng.uniform(0.02, 1.0, (256, 3)) @ np.array([[0.4124, 0.3576, 0.1805], [0.2126, 0.7152, 0.0722],
                                                        [0.0193, 0.1192, 0.9505]]).T
    xyy = np.stack([inner[:, 0] / inner.sum(1), inner[:, 1] / inner.sum(1), inner[:, 1]], axis=1)
    inputs = np.stack([rgb, rgb, inner, xyy]).astype(np.float32)          # [colour space][256][3]
    packed = np.zeros((4, 4, 256, 3), np.uint32)
    for t in range(4):
        for c in range(4):
            for i in range(256):
                packed[t, c, i] = ref.upsample(t, c, *map(float, inputs[c, i]))
    np.savez_compressed(os.path.join(HERE, "upsample.npz"), inputs=inputs, packed=packed)

    W = H = 32
    spp = 256
    desc = scenes.cornell_box_desc(W, H)
    film, _, seg = ref.pt_render(scenes.flatten_desc(desc), desc["camera"], W, H, spp, 8)
    _, _, cmf, _ = ref.tables()
    y = np.einsum("hwk,k->hw", film, cmf[1].astype(np.float64))
    np.savez_compressed(os.path.join(HERE, "pt_cornell_32.npz"), y=y, spp=spp, segments=seg)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
