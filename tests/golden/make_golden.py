"""Generate the golden vectors of ``tests/golden/*.npz``.

Runs the REFERENCE engine (leviathan_kernel.cu built from the reference's own
sources by ``oracle/Makefile``, on a CUDA device) over seeded fixtures
through its C ABI, exactly as its pybind binding and LeviathanObservatory
drive it (python/leviathan_h100.py:82-93, 198-207), and stores inputs and
outputs.  These files pin ``oracle/oracle64.py`` and the B200 engine.

    python tests/golden/make_golden.py --out tests/golden            # GPU
    python tests/golden/make_golden.py --engine oracle --out /tmp/x  # dry run

Each case is a list of actions replayed identically by the tests:
("step", n) -> n calls of step(dt); ("set_theta", kick) -> get_theta,
add kick, wrap mod 2pi (or write NaN/inf), set_theta; ("set_gain", g);
("controller", on).
"""

from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from leviathan_v1_b200.graphs import config_small, init_state, make_network  # noqa: E402

DT = 0.05


def case_c0():
    net = config_small(0)
    actions = [("step", 500)]
    record = dict(theta=[1, 10, 100, 150, 199, 200, 500],
                  weights=[200, 500], predictor=[200, 500], ring=[200])
    return net, actions, record


def case_tiny():
    net = make_network(200, 8, 0.1, 10, 1, delay_lo=0, delay_hi=10)
    actions = [("step", 200)]
    record = dict(theta=[1, 2, 3, 10, 100, 200], weights=[1, 10, 200],
                  predictor=[200], ring=[10, 200])
    return net, actions, record


def case_edge():
    """Ragged CSR: empty rows, one hub row of 5000 (repeated) sources,
    delays in [0, max_delay]; a stimulus, a gain override and the
    controller switched off midway."""
    rng = np.random.default_rng(7)
    N, max_delay = 300, 7
    deg = rng.integers(0, 12, N)
    deg[rng.choice(N, 25, replace=False)] = 0
    deg[123] = 5000
    row_ptr = np.zeros(N + 1, np.int64)
    np.cumsum(deg, out=row_ptr[1:])
    E = int(row_ptr[-1])
    col = rng.integers(0, N, E).astype(np.int32)
    row_ptr = row_ptr.astype(np.int32)
    st = init_state(row_ptr, max_delay, 11, delay_lo=0, delay_hi=max_delay)
    from leviathan_v1_b200.graphs import Network

    net = Network(N, max_delay, row_ptr, col, st["delays"], st["weights"],
                  st["theta"], st["theta_hat"], st["omega"])
    kick = np.zeros(N, np.float32)
    kick[:10] = 2.0
    actions = [("step", 30), ("set_theta", kick), ("step", 30),
               ("set_gain", 2.5), ("controller", False), ("step", 40)]
    record = dict(theta=[1, 30, 31, 60, 100], weights=[1, 30, 60, 100],
                  predictor=[100], ring=[31, 100])
    return net, actions, record


def case_nan():
    net = make_network(200, 8, 0.1, 12, 3)
    bad = np.zeros(200, np.float32)
    bad[5] = np.nan
    bad[7] = np.inf
    actions = [("step", 10), ("set_theta_raw", bad), ("step", 40)]
    record = dict(theta=[10, 11, 12, 50], weights=[11, 12, 50],
                  predictor=[12, 50], ring=[50])
    return net, actions, record


def case_sweep():
    net = make_network(500, 16, 0.1, 20, 5)
    actions = [("controller", False), ("set_gain", 3.0), ("step", 100)]
    record = dict(theta=[100], weights=[100], predictor=[100], ring=[100])
    return net, actions, record


CASES = dict(c0=case_c0, tiny=case_tiny, edge=case_edge, nan=case_nan,
             sweep=case_sweep)


class _OracleAdapter:
    """Dry-run stand-in with the RefEngine interface (oracle, FP32)."""

    def __init__(self, *args):
        sys.path.insert(0, os.path.join(REPO, "oracle"))
        from oracle64 import OracleEngine

        self.o = OracleEngine(*args, dtype=np.float32)

    def step(self, dt):
        return self.o.step(dt)

    def get_theta(self):
        return self.o.get_theta().astype(np.float32)

    def set_theta(self, t):
        self.o.set_theta(t)

    def set_gain(self, g):
        self.o.set_gain(g)

    def set_gain_controller(self, on):
        self.o.set_gain_controller(on)

    def state(self):
        o = self.o
        return dict(theta=o.theta.astype(np.float32),
                    theta_hat=o.theta_hat.astype(np.float32),
                    omega_hat=o.omega_hat.astype(np.float32),
                    weights=o.w.astype(np.float32), ring=o.ring.astype(np.float32),
                    buf_idx=o.buf_idx, g=float(o.g))

    def close(self):
        pass


def replay(engine, actions, record, dt=DT):
    """Apply ``actions``; return r(t) and the recorded snapshots."""
    rs, out, t = [], {}, 0
    want = {k: set(v) for k, v in record.items()}

    def snap():
        s = engine.state()
        if t in want.get("theta", ()):
            out[f"theta@{t}"] = s["theta"]
        if t in want.get("weights", ()):
            out[f"weights@{t}"] = s["weights"]
        if t in want.get("predictor", ()):
            out[f"theta_hat@{t}"] = s["theta_hat"]
            out[f"omega_hat@{t}"] = s["omega_hat"]
        if t in want.get("ring", ()):
            out[f"ring@{t}"] = s["ring"]
            out[f"buf_idx@{t}"] = np.int32(s["buf_idx"])
        out[f"g@{t}"] = np.float32(s["g"])

    for act in actions:
        kind = act[0]
        if kind == "step":
            for _ in range(act[1]):
                rs.append(engine.step(dt))
                t += 1
                if any(t in v for v in want.values()):
                    snap()
        elif kind == "set_theta":
            th = engine.get_theta()
            th = (th + act[1]) % np.float32(2 * np.pi)
            engine.set_theta(th.astype(np.float32))
        elif kind == "set_theta_raw":
            th = engine.get_theta()
            m = act[1] != 0
            th = th.copy()
            th[m] = act[1][m]
            engine.set_theta(th.astype(np.float32))
        elif kind == "set_gain":
            engine.set_gain(act[1])
        elif kind == "controller":
            engine.set_gain_controller(act[1])
        else:
            raise ValueError(kind)
    return np.array(rs, np.float32), out


def encode_actions(actions):
    """Actions as arrays for the npz (kinds, scalar args, vector args)."""
    kinds, scal, vecs = [], [], []
    for a in actions:
        kinds.append(a[0])
        if a[0] in ("set_theta", "set_theta_raw"):
            scal.append(len(vecs))
            vecs.append(np.asarray(a[1], np.float32))
        elif a[0] == "controller":
            scal.append(1.0 if a[1] else 0.0)
        else:
            scal.append(float(a[1]))
    return np.array(kinds), np.array(scal, np.float64), vecs


def decode_actions(z):
    kinds = [str(k) for k in z["action_kind"]]
    scal = z["action_arg"]
    out = []
    for k, a in zip(kinds, scal):
        if k in ("set_theta", "set_theta_raw"):
            out.append((k, z[f"action_vec{int(a)}"]))
        elif k == "controller":
            out.append((k, bool(a)))
        elif k == "step":
            out.append((k, int(a)))
        else:
            out.append((k, float(a)))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--engine", choices=["reference", "oracle"], default="reference")
    ap.add_argument("--flavor", default="sm100a")
    ap.add_argument("--cases", default=",".join(CASES))
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    for name in args.cases.split(","):
        net, actions, record = CASES[name]()
        if args.engine == "reference":
            sys.path.insert(0, os.path.join(REPO, "oracle"))
            from refengine import RefEngine

            eng = RefEngine(*net.engine_args(), flavor=args.flavor)
        else:
            eng = _OracleAdapter(*net.engine_args())
        rs, snaps = replay(eng, actions, record)
        eng.close()
        kinds, scal, vecs = encode_actions(actions)
        payload = dict(N=net.N, max_delay=net.max_delay, row_ptr=net.row_ptr,
                       col_idx=net.col_idx, delays=net.delays, weights=net.weights,
                       theta=net.theta, theta_hat=net.theta_hat, omega=net.omega,
                       dt=np.float32(DT), r=rs, action_kind=kinds, action_arg=scal,
                       engine=np.array(f"{args.engine}:{args.flavor}"))
        for i, v in enumerate(vecs):
            payload[f"action_vec{i}"] = v
        payload.update(snaps)
        path = os.path.join(args.out, f"{name}.npz")
        np.savez_compressed(path, **payload)
        print(f"{name}: N={net.N} E={net.E} steps={rs.size} r[-1]={rs[-1]:.6f} -> {path}")


if __name__ == "__main__":
    main()
