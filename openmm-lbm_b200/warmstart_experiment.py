"""Runs the learned warm-start experiment (warmstart.main): steady solves of obstacle channels for training and
held-out seeds, training of the U-Net on the tensor-core convolutions, and warm against cold solves of the held-out
seeds.  The package is loaded from this folder.

    python openmm-lbm_b200/warmstart_experiment.py --train 2000 --test 200 --epochs 8 --out report.json
"""
import importlib.util
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def load_package():
    if 'lbm_b200' not in sys.modules:
        spec = importlib.util.spec_from_file_location('lbm_b200', os.path.join(HERE, '__init__.py'),
                                                      submodule_search_locations=[HERE])
        module = importlib.util.module_from_spec(spec)
        sys.modules['lbm_b200'] = module
        spec.loader.exec_module(module)
    return sys.modules['lbm_b200']


if __name__ == '__main__':
    load_package()
    from lbm_b200 import warmstart
    warmstart.main()
