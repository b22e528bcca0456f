"""Trains the warm-start network of the obstacle channel (128x64x64, 5-20 spheres of radius 4-10, Velocity inlet 0.02,
Density outlet, tau 0.6) on steady states that the plain solver computes, and writes it to weights.pt in this folder,
where bench.py's time-to-steady measurement and the tests load it.  Needs a GPU; a few minutes per thousand training
channels.

    python openmm-lbm_b200/warmstart_net/train.py [--train 1000 --epochs 16 --test 16] [--to DIR]

Training seeds 1..train, held-out seeds 100001..; the report (loss history, held-out speed-ups) goes to report.json
beside the weights.  --to writes both to another folder (copy them here afterwards).
"""
import importlib.util
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PACKAGE = os.path.dirname(HERE)


def load_package():
    if 'lbm_b200' in sys.modules:
        return sys.modules['lbm_b200']
    spec = importlib.util.spec_from_file_location('lbm_b200', os.path.join(PACKAGE, '__init__.py'),
                                                  submodule_search_locations=[PACKAGE])
    module = importlib.util.module_from_spec(spec)
    sys.modules['lbm_b200'] = module
    spec.loader.exec_module(module)
    return module


if __name__ == '__main__':
    load_package()
    from lbm_b200 import warmstart
    args = sys.argv[1:]
    out = HERE
    if '--to' in args:
        i = args.index('--to')
        out = args[i + 1]
        del args[i:i + 2]
        os.makedirs(out, exist_ok=True)
    defaults = {'--train': '1000', '--epochs': '16', '--test': '16'}
    for k, v in defaults.items():
        if k not in args:
            args += [k, v]
    warmstart.main(args + ['--save', os.path.join(out, 'weights.pt'), '--out', os.path.join(out, 'report.json'),
                           '--no-conv-benchmark'])
