"""Command-line front end with the reference CLI's flags and rules
(cli/src/main.rs:8-144):

    python -m rtrace_b200 -i scene.json -o out.png [-s 1000] [--max-depth 10]
                          [--samples N] [--anti-aliasing quincunx|stochastic|no-jitter]

The image size comes from the diagonal -s and the camera's width/height
ratio (H = D / sqrt(R^2 + 1), W = R * H, each rounded half away from zero);
the seed is always 0; a scene with outlines enabled switches quincunx to
no-jitter.  Rendering runs on the GPU.
"""
import argparse
import math
import os
import sys


def image_size(aspect, diagonal):
    """cli/src/main.rs:339-350"""
    h = diagonal / math.sqrt(aspect * aspect + 1.0)
    w = aspect * h
    return round_u32(w), round_u32(h)


def round_u32(v):
    """`v.round() as u32`: half away from zero, then a saturating cast."""
    if not v > 0:  # NaN and negatives saturate to 0
        return 0
    if v >= 4294967295.0:
        return 4294967295
    q = math.floor(v)
    return int(q + 1 if v - q >= 0.5 else q)


def main(argv=None):
    ap = argparse.ArgumentParser(prog="rtrace", description="Ray tracer CLI - renders 3D scenes from JSON descriptions")
    ap.add_argument("-i", "--input", required=True)
    ap.add_argument("-o", "--output", required=True)
    ap.add_argument("-s", "--size", type=int, default=1000)
    ap.add_argument("--max-depth", type=int, default=10)
    ap.add_argument("--samples", type=int, default=None)
    ap.add_argument("--anti-aliasing", default="quincunx")
    a = ap.parse_args(argv)
    import rtrace_b200 as rt
    if not os.path.exists(a.input):
        print("Error: Input file '%s' does not exist" % a.input, file=sys.stderr)
        return 1
    modes = {"quincunx": rt.AntiAliasingMode.Quincunx, "stochastic": rt.AntiAliasingMode.Stochastic,
             "no-jitter": rt.AntiAliasingMode.NoJitter}
    if a.anti_aliasing not in modes:
        print("Error: Invalid anti-aliasing mode '%s'. Valid options are: quincunx, stochastic, no-jitter"
              % a.anti_aliasing, file=sys.stderr)
        return 1
    samples = a.samples if a.samples is not None else 1
    if samples == 0:
        print("Error: Samples must be greater than 0", file=sys.stderr)
        return 1
    try:
        scene = rt.Scene.from_json_file(a.input)
    except rt.RtraceError as e:
        print("Error loading scene from '%s': %s" % (a.input, e), file=sys.stderr)
        return 1
    w, h = image_size(scene.camera_aspect, float(a.size))
    r = rt.Renderer(w, h)
    r.max_depth = a.max_depth
    r.samples = samples
    r.seed = 0
    mode = modes[a.anti_aliasing]
    try:
        oc = scene.get_outline_config()
    except rt.RtraceError as e:
        print("Error: Invalid outline color in scene: %s" % e, file=sys.stderr)
        return 1
    if oc is not None:
        r.with_outline_detection(oc)
        if mode == rt.AntiAliasingMode.Quincunx:
            print("Warning: Quincunx anti-aliasing is not compatible with outline detection. "
                  "Switching to no-jitter mode.")
            mode = rt.AntiAliasingMode.NoJitter
    r.anti_aliasing_mode = mode
    try:
        r.render_to_file(scene, a.output)
    except (rt.RtraceError, ValueError) as e:
        print("Error rendering image: %s" % e, file=sys.stderr)
        return 1
    print("Successfully rendered to '%s'" % a.output)
    return 0


if __name__ == "__main__":
    sys.exit(main())
