"""Loading the golden fixtures made by tests/golden/make_golden.py."""
import json
import os

import numpy as np

from grappolo_b200.graphs import CSRGraph

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')
CASES = ['karate', 'pp1000', 'pp1000_w', 'rmat10', 'pair', 'loops_isolated', 'cycle4_ties',
         'hubs', 'hubs_w']


def load(name):
    z = dict(np.load(os.path.join(GOLDEN, f'{name}.npz')))
    g = CSRGraph(z['ptr'], z['tail'], z['weight'])
    return g, z


def pins():
    with open(os.path.join(GOLDEN, 'pins.json')) as f:
        return json.load(f)
