"""Helpers shared by the test modules."""

from __future__ import annotations

import types
from pathlib import Path

import numpy as np

import lbm_b200 as lbm

GOLDEN = Path(__file__).resolve().parent / "golden"

NS = types.SimpleNamespace(
    SimulationParams=lbm.SimulationParams, channel_walls=lbm.channel_walls, cavity_walls=lbm.cavity_walls,
    circle=lbm.circle, sphere=lbm.sphere, voxelize=lbm.voxelize, wall_links=lbm.wall_links,
    ImmersedBoundary=lbm.ImmersedBoundary, default_lattice=lbm.default_lattice, LinkRules=lbm.LinkRules,
    bouzidi_rules=lbm.bouzidi_rules, open_channel=lbm.open_channel,
)
"""This package's builders, in the shape ``tests/cases.py`` expects."""


def reference_ns():
    """The reference's own builders (the unmodified package in baseline/_ref), in the shape
    ``tests/cases.py`` expects; None where it is not installed."""
    from oracle import reference_package

    ref = reference_package.modules()
    if ref is None:
        return None
    from lbm.boundaries import cavity_walls, channel_walls  # noqa: PLC0415

    g, lk = ref.geometry, ref.link_rules
    return types.SimpleNamespace(
        SimulationParams=ref.params.SimulationParams, channel_walls=channel_walls, cavity_walls=cavity_walls,
        circle=g.circle, sphere=g.sphere, voxelize=g.voxelize, wall_links=g.wall_links,
        ImmersedBoundary=ref.ibm.ImmersedBoundary, default_lattice=ref.lattice.default_lattice,
        LinkRules=lk.LinkRules, bouzidi_rules=lk.bouzidi_rules, open_channel=ref.open_boundaries.open_channel,
    )


def golden(name: str) -> dict:
    with np.load(GOLDEN / f"{name}.npz") as data:
        return {k: data[k] for k in data.files}


def rule_map(node, direction, tdir, tnode, coeff, const):
    """{(node, direction): (const, {(k, y): coeff})} with zero terms dropped."""
    out = {}
    for r in range(len(node)):
        terms = {}
        for k, y, a in zip(tdir[r], tnode[r], coeff[r], strict=True):
            if a != 0.0:
                terms[(int(k), int(y))] = terms.get((int(k), int(y)), 0.0) + float(a)
        out[(int(node[r]), int(direction[r]))] = (float(const[r]), terms)
    return out


def assert_rules_match(ours, ref: dict, prefix: str, atol=1e-14):
    """Compare a LinkRules with golden arrays (set of links, constants and terms)."""
    v = ours.values
    mine = rule_map(ours.node, ours.direction, v.direction, v.node, v.coeff, v.constant)
    theirs = rule_map(ref[f"{prefix}node"], ref[f"{prefix}direction"], ref[f"{prefix}tdir"], ref[f"{prefix}tnode"],
                      ref[f"{prefix}coeff"], ref[f"{prefix}const"])
    assert mine.keys() == theirs.keys()
    for key, (const, terms) in theirs.items():
        c2, t2 = mine[key]
        assert abs(c2 - const) <= atol, (key, c2, const)
        keys = {k for k, a in terms.items() if abs(a) > atol} | {k for k, a in t2.items() if abs(a) > atol}
        for k in keys:
            assert abs(terms.get(k, 0.0) - t2.get(k, 0.0)) <= atol, (key, k)
    # the rule order is part of the contract for force probes built on them
    np.testing.assert_array_equal(ours.node, ref[f"{prefix}node"])
    np.testing.assert_array_equal(ours.direction, ref[f"{prefix}direction"])
