"""Step one seeded scene on the GPU world and exit (profiling driver).

  python -m melon3d_b200.harness <scene> [--steps N] [--seed S] [-a A -b B -c C] [--giant CONTACTS]

Scenes: pyramid, rain, pile, raft, batch_world, incline, jointed_raft,
settled_stacks (parameters a, b, c as in scenes.cpp).  Used by the ncu
commands recorded under profiles/: the same command line runs once plain and
once under ncu.
"""
import argparse
import sys

from .. import api
from . import (BATCH_WORLD, INCLINE, JOINTED_RAFT, PILE, PYRAMID, RAFT, RAIN, SETTLED_STACKS, Scene)

SCENES = {"pyramid": PYRAMID, "rain": RAIN, "pile": PILE, "raft": RAFT, "batch_world": BATCH_WORLD,
          "incline": INCLINE, "jointed_raft": JOINTED_RAFT, "settled_stacks": SETTLED_STACKS}


def main(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("scene", choices=sorted(SCENES))
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--seed", type=int, default=1)
    p.add_argument("-a", type=int, default=0)
    p.add_argument("-b", type=int, default=0)
    p.add_argument("-c", type=int, default=0)
    p.add_argument("--giant", type=int, default=0, help="giant-island contact threshold (0: the default)")
    args = p.parse_args(argv)
    lib = api.load_gpu()
    sc = Scene(lib, SCENES[args.scene], args.seed, args.a, args.b, args.c)
    if args.giant > 0:
        lib.m3d_gpu_set_giant_island_contacts(sc.world, args.giant)
    sc.run(args.steps)
    status = lib.m3d_gpu_status(sc.world)
    pr = lib.m3d_world_profile(sc.world)
    print("%s: %d steps, bodies %d, contacts %d, touching %d, status %d" % (
        args.scene, args.steps, pr.bodyCount, pr.contactCount, pr.touchingContactCount, status))
    sc.close()
    return 0 if status == api.GPU_OK else 1


if __name__ == "__main__":
    sys.exit(main())
