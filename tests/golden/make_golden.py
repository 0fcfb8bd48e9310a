"""Generate golden vectors from the unmodified reference package.

Run in a checkout that has the reference's sources (pure Python + NumPy)::

    python tests/golden/make_golden.py /path/to/reference/src

It imports the reference's ``lbm`` package, builds the cases of
``tests/cases.py`` with the reference's own builders, runs its NumPy
``ReferenceSolver`` and writes one compressed ``.npz`` per case next to this
script. The fixtures pin the oracle (``oracle/``) and this package's host-side
builders; the GPU never needs the reference.
"""

from __future__ import annotations

import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))


def reference_namespace(src: str):
    sys.path.insert(0, src)
    from lbm import SimulationParams, make_solver  # noqa: PLC0415
    from lbm.boundaries import cavity_walls, channel_walls
    from lbm.forces import ForceProbe
    from lbm.geometry import circle, sphere, voxelize, wall_links
    from lbm.ibm import ImmersedBoundary
    from lbm.lattice import default_lattice
    from lbm.link_rules import LAYOUTS, LinkRules, bouzidi_rules, compile_affine, compile_rules
    from lbm.open_boundaries import open_channel
    from lbm.solver import SimulationDiverged

    return types.SimpleNamespace(
        SimulationParams=SimulationParams, make_solver=make_solver, channel_walls=channel_walls,
        cavity_walls=cavity_walls, circle=circle, sphere=sphere, voxelize=voxelize,
        wall_links=wall_links, ImmersedBoundary=ImmersedBoundary, default_lattice=default_lattice,
        LinkRules=LinkRules, bouzidi_rules=bouzidi_rules, compile_affine=compile_affine, compile_rules=compile_rules,
        open_channel=open_channel, ForceProbe=ForceProbe, LAYOUTS=LAYOUTS,
        SimulationDiverged=SimulationDiverged,
    )


def rules_arrays(prefix, rules):
    v = rules.values
    return {
        f"{prefix}node": np.asarray(rules.node), f"{prefix}direction": np.asarray(rules.direction),
        f"{prefix}tdir": np.asarray(v.direction), f"{prefix}tnode": np.asarray(v.node),
        f"{prefix}coeff": np.asarray(v.coeff), f"{prefix}const": np.asarray(v.constant),
    }


def run(ns, params, state, steps):
    solver = ns.make_solver(params, backend="numpy")
    if state is not None:
        solver.initialize(*state)
    solver.run(steps)
    return solver


def outputs(solver, d):
    m = solver.macroscopic()
    out = {"f": solver.populations(), "rho": np.asarray(m.rho)}
    for a in range(d):
        out[f"u{a}"] = np.asarray(m.u[a])
    return out


def main(src: str) -> None:
    from tests import cases

    ns = reference_namespace(src)
    steps = cases.EQUIVALENCE_STEPS
    written = []

    def save(name, **arrays):
        path = HERE / f"{name}.npz"
        np.savez_compressed(path, **arrays)
        written.append((name, path.stat().st_size))

    # mixed geometry: walls, moving lid/plate, obstacle, force
    for d, size in ((2, None), (3, (15, 13, 11))):
        for dtype, collision in (("float64", "trt"), ("float64", "bgk"), ("float32", "trt")):
            p = cases.mixed(ns, dtype, collision, d, size)
            s = run(ns, p, cases.random_state(p), steps)
            save(f"mixed{d}d_{dtype}_{collision}", steps=steps, **outputs(s, d))

    # Bouzidi body + force probe in every layout
    for d, size, body in ((2, None, None), (3, (16, 14, 12), ns.sphere(7.3, 6.6, 5.8, 3.1))):
        for dtype in ("float64", "float32"):
            p, links = cases.bouzidi(ns, d, dtype, size, body)
            s = run(ns, p, cases.random_state(p), steps)
            probe = ns.ForceProbe.build(p, links)
            extra = {"probe_force": probe.evaluate(s), "probe_weight": probe.weight}
            extra |= rules_arrays("probe_", types.SimpleNamespace(node=np.zeros(0), direction=np.zeros(0), values=probe.values))
            for layout in ("pull", "aa_odd", "aa_even"):
                comp = probe.compiled(layout)
                extra |= {f"{layout}_slots": comp.slots, f"{layout}_coeff": comp.coeff, f"{layout}_const": comp.constant}
            save(
                f"bouzidi{d}d_{dtype}", steps=steps, link_node=links.node, link_dir=links.direction,
                link_q=links.q, **rules_arrays("rule_", p.link_rules), **extra, **outputs(s, d),
            )

    # IBM body
    for d, size, body in ((2, None, None), (3, (14, 14, 12), ns.sphere(6.7, 6.6, 5.9, 2.6))):
        for dtype in ("float64", "float32"):
            p = cases.ibm(ns, d, dtype, size, body)
            s = run(ns, p, cases.random_state(p), steps)
            nodes, weights = p.immersed.stencil(p.shape)
            save(
                f"ibm{d}d_{dtype}", steps=steps, markers=p.immersed.markers, areas=p.immersed.areas,
                stencil_nodes=nodes, stencil_weights=weights, immersed_force=s.immersed_force,
                **outputs(s, d),
            )

    # Zou-He open channel
    for d in (2, 3):
        p, inflow = cases.open_channel_case(ns, d)
        s = run(ns, p, cases.random_state(p, seed=1, u_scale=0.03), steps)
        save(f"zouhe{d}d_float64", steps=steps, solid=p.solid, **rules_arrays("rule_", p.link_rules), **outputs(s, d))

    # Link rules compiled to the pre-pass slots of every layout (the reference's
    # compile_rules), for the cases the GPU checker runs against the reference's
    # own rule pre-pass kernels
    compiled = {}
    for d in (2, 3):
        for name, (p, _) in (("bouzidi", cases.bouzidi(ns, d, "float64")),
                             ("zouhe", cases.open_channel_case(ns, d))):
            for layout in ("pull", "aa_odd", "aa_even"):
                c = ns.compile_rules(p.lattice, p.link_rules, layout, p.solid, p.wall_velocity)
                key = f"{name}{d}d_{layout}_"
                compiled |= {key + "target": np.asarray(c.target), key + "slots": np.asarray(c.values.slots),
                             key + "coeff": np.asarray(c.values.coeff), key + "const": np.asarray(c.values.constant)}
    save("compiled_rules", **compiled)

    # Configuration geometries: rule builders only (no run)
    p, links, _ = cases.cylinder_channel(ns, "bouzidi")
    save("cylinder_bouzidi_rules", solid=p.solid, link_node=links.node, link_dir=links.direction,
         link_q=links.q, **rules_arrays("rule_", p.link_rules))
    p, _, _ = cases.cylinder_channel(ns, "ibm")
    nodes, weights = p.immersed.stencil(p.shape)
    save("cylinder_ibm_markers", markers=p.immersed.markers, areas=p.immersed.areas,
         stencil_nodes=nodes, stencil_weights=weights, **rules_arrays("rule_", p.link_rules))
    p, links, _ = cases.sphere_channel(ns, nx=40, ny=20, nz=18, radius=4.0)
    save("sphere_channel_small_rules", solid=p.solid, link_node=links.node, link_dir=links.direction,
         link_q=links.q, **rules_arrays("rule_", p.link_rules))

    # Configurations at reduced size, run by the reference
    p, state = cases.tgv(ns, n=64)
    s = run(ns, p, state, 200)
    save("tgv64_float32", steps=200, **outputs(s, 2))
    for dtype in ("float64", "float32"):
        p = cases.duct(ns, n=18, nx=4, dtype=dtype, force=1e-5)
        s = run(ns, p, None, 200)
        save(f"duct18_{dtype}", steps=200, **outputs(s, 3))
    p = cases.cavity(ns, 30, 400.0, dtype="float64")
    s = run(ns, p, None, 300)
    save("cavity30_float64", steps=300, **outputs(s, 2))

    # Watchdog: where and when a NaN is reported
    for d in (2, 3):
        sizes = {"nx": 8, "ny": 8} | ({"nz": 8} if d == 3 else {})
        p = ns.SimulationParams(**sizes, tau=0.8, dtype="float64")
        solver = ns.make_solver(p, backend="numpy")
        rho = np.ones(p.shape)
        rho[(3, 5, 2)[:d]] = np.nan
        solver.initialize(rho)
        try:
            solver.run(10, check_every=5)
            raise AssertionError("expected divergence")
        except ns.SimulationDiverged as exc:
            save(f"watchdog{d}d", step=exc.step, location=np.asarray(exc.location), message=str(exc))

    for name, size in written:
        print(f"{name:32s} {size / 1024:8.1f} KiB")
    print(f"total {sum(s for _, s in written) / 2**20:.2f} MiB")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference/src")
