"""Seeded generators for the benchmark networks, written as UPPAAL XML in the
subset the reference front end accepts (so the same file runs through the
reference binary and through this library).

* :func:`random_network` — small random networks (8 components x 4 locations
  x 6 edges, one clock each, two shared ints, one broadcast channel).
* :func:`epidemic` — agent-based SEIR epidemic over shared counters, infection
  rate beta*I/N per susceptible, infections announced on a broadcast channel.
* :func:`mutex` — Fischer-style timed mutual exclusion with n processes.
* :func:`batch_networks` — many random networks of uneven size for batched runs.

Generated models avoid the constructs that make the reference kernel
misbehave: every location is reachable from its initial location (the
reference's upload needs every node, shared_model_state.cu:475), at most one
receiving edge per location (a receiver with several enabled edges uses an
invalid random state pointer, simulation.cu:385), and every location with a
clock invariant ends its edge list with an always-enabled, clock-resetting
edge, so a component that reaches its bound leaves it instead of proposing a
zero delay forever.
"""
from __future__ import annotations

import math
import random
from dataclasses import dataclass
from xml.sax.saxutils import escape


@dataclass
class Workload:
    """A generated network and the query the benchmark asks of it."""

    name: str
    xml: str
    var_id: int          # tracked variable (-1: location query)
    threshold: int       # probability query: max > threshold
    horizon: int
    runs: int
    loc_query: str = ""
    is_max: bool = True
    is_estimate: bool = False
    n_vars: int = 0      # int and clock variables the network declares (what the
                         # reference's variable registry counts; 0: not recorded)

    def cli_query(self) -> list[str]:
        """The reference CLI's -q arguments for this workload."""
        return ["-q", str(self.runs), str(self.horizon), str(self.threshold), str(self.var_id),
                "1" if self.is_max else "0", "1" if self.is_estimate else "0", self.loc_query]

    def write(self, path: str) -> str:
        with open(path, "w") as f:
            f.write(self.xml)
        return path


def _label(kind: str, text: str) -> str:
    return f'<label kind="{kind}">{escape(text)}</label>'


class _Doc:
    def __init__(self, global_decl: str):
        self.parts = ['<?xml version="1.0" encoding="utf-8"?>', "<nta>",
                      f"<declaration>{escape(global_decl)}</declaration>"]
        self.next_id = 0

    def new_id(self) -> str:
        i = self.next_id
        self.next_id += 1
        return f"id{i}"

    def template(self, name: str, local_decl: str, locations, init_ref: str, transitions) -> None:
        p = self.parts
        p.append("<template>")
        p.append(f"<name>{escape(name)}</name>")
        p.append(f"<declaration>{escape(local_decl)}</declaration>")
        for loc_id, loc_name, labels in locations:
            p.append(f'<location id="{loc_id}">')
            if loc_name:
                p.append(f"<name>{escape(loc_name)}</name>")
            for kind, text in labels:
                p.append(_label(kind, text))
            p.append("</location>")
        p.append(f'<init ref="{init_ref}"/>')
        for src, dst, labels in transitions:
            p.append("<transition>")
            p.append(f'<source ref="{src}"/>')
            p.append(f'<target ref="{dst}"/>')
            for kind, text in labels:
                p.append(_label(kind, text))
            p.append("</transition>")
        p.append("</template>")

    def finish(self) -> str:
        self.parts.append("<system>system;</system>")
        self.parts.append("</nta>")
        return "\n".join(self.parts) + "\n"


def epidemic(n_agents: int = 100, beta: float = 0.3, rate_ei: float = 0.2, rate_ir: float = 0.1,
             r_threshold: int = 50, horizon: int = 100, runs: int = 1_000_000) -> Workload:
    """SEIR agents over shared counters S, E, I, R (variable ids 0..3); agent 0
    starts infected.  Query Pr[<=T](<> R >= r_threshold)."""
    decl = "\n".join([
        f"const int N = {n_agents};",
        f"const double beta = {beta};",
        f"int S = {n_agents - 1};",
        "int E = 0;",
        "int I = 1;",
        "int R = 0;",
        "broadcast chan inf;",
    ])
    d = _Doc(decl)
    for k in range(n_agents):
        # the index case starts infected; it has no S and E locations, which
        # would be unreachable from its initial location
        s, e = (None, None) if k == 0 else (d.new_id(), d.new_id())
        i, r = d.new_id(), d.new_id()
        locs = []
        trans = []
        if k:
            locs += [(s, "S", [("exponentialrate", "beta * I / N")]),
                     (e, "E", [("exponentialrate", f"{rate_ei}")])]
            trans += [(s, e, [("synchronisation", "inf!"), ("assignment", "S = S - 1, E = E + 1")]),
                      (e, i, [("assignment", "E = E - 1, I = I + 1")])]
        locs += [(i, "I", [("exponentialrate", f"{rate_ir}")]), (r, "R", [])]
        trans += [(i, r, [("assignment", "I = I - 1, R = R + 1")])]
        d.template(f"Agent{k}", "", locs, i if k == 0 else s, trans)
    return Workload(f"epidemic_{n_agents}", d.finish(), var_id=3, threshold=r_threshold - 1, horizon=horizon,
                    runs=runs, n_vars=4)


def mutex(n: int = 32, k: int = 2, horizon: int = 200, runs: int = 10_000_000) -> Workload:
    """Fischer-style mutual exclusion: shared id (var 0) and a counter of
    processes in the critical section (var 1).  Query Pr[<=T](<> incs >= 2)."""
    decl = "\n".join(["int id = 0;", "int incs = 0;", f"const int k = {k};"])
    d = _Doc(decl)
    for p in range(n):
        idle, req, wait, cs = d.new_id(), d.new_id(), d.new_id(), d.new_id()
        locs = [
            (idle, "idle", [("exponentialrate", "1")]),
            (req, "req", [("invariant", "x <= k")]),
            (wait, "wait", []),
            (cs, "cs", [("exponentialrate", "1")]),
        ]
        trans = [
            (idle, req, [("guard", "id == 0"), ("assignment", "x = 0")]),
            (req, wait, [("assignment", "x = 0, id = pid")]),
            (wait, cs, [("guard", "x > k && id == pid"), ("assignment", "incs = incs + 1")]),
            (wait, idle, [("guard", "id == 0")]),
            (cs, idle, [("assignment", "id = 0, incs = incs - 1")]),
        ]
        d.template(f"P{p}", f"clock x;\nconst int pid = {p + 1};", locs, idle, trans)
    return Workload(f"mutex_{n}", d.finish(), var_id=1, threshold=1, horizon=horizon, runs=runs, n_vars=2 + n)


def random_network(seed: int, n_comps: int = 8, n_locs: int = 4, n_edges: int = 6, horizon: int = 100,
                   runs: int = 10_000, target: int = 8) -> Workload:
    """Random network of clocked automata over two shared ints v0, v1 in
    [0, 16].  Query Pr[<=T](<> v0 >= target)."""
    rng = random.Random(seed)
    v0, v1 = rng.randint(0, 16), rng.randint(0, 16)
    d = _Doc(f"int v0 = {v0};\nint v1 = {v1};\nbroadcast chan bc;")
    for c in range(n_comps):
        ids = [d.new_id() for _ in range(n_locs)]
        order = list(range(n_locs))
        rng.shuffle(order)
        # a cycle through all locations keeps every location reachable and
        # gives each one an outgoing edge; the rest are random
        edges = [(order[j], order[(j + 1) % n_locs]) for j in range(n_locs)]
        for _ in range(max(0, n_edges - n_locs)):
            edges.append((rng.randrange(n_locs), rng.randrange(n_locs)))
        spine = {order[j]: j for j in range(n_locs)}  # edge index of each location's cycle edge
        lows = {j: rng.randint(0, 10) for j in range(len(edges))}
        max_low = {l: max(lows[j] for j, (s, _) in enumerate(edges) if s == l) for l in range(n_locs)}
        invariant = {l: rng.random() < 0.5 for l in range(n_locs)}
        bounds = {l: rng.randint(max_low[l] + 1, max(max_low[l] + 1, 20)) for l in range(n_locs)}
        locs = []
        for l in range(n_locs):
            if invariant[l]:
                locs.append((ids[l], f"L{l}", [("invariant", f"x <= {bounds[l]}")]))
            else:
                lam = math.exp(rng.uniform(math.log(0.1), math.log(2.0)))
                locs.append((ids[l], f"L{l}", [("exponentialrate", f"{lam:.4f}")]))
        trans_by_src: dict[int, list] = {l: [] for l in range(n_locs)}
        receivers = set()
        for j, (s, t) in enumerate(edges):
            guards = [f"x >= {lows[j]}"]
            labels = []
            escape_edge = invariant[s] and j == spine[s]
            ups = []
            if escape_edge:
                ups.append("x = 0")
                if rng.random() < 0.1:
                    labels.append(("synchronisation", "bc!"))
            else:
                var = rng.choice(["v0", "v1"])
                delta = rng.choice([-1, 0, 1])
                if delta == -1:
                    guards.append(f"{var} >= 1")
                    ups.append(f"{var} = {var} - 1")
                elif delta == 1:
                    guards.append(f"{var} <= 15")
                    ups.append(f"{var} = {var} + 1")
                if rng.random() < 0.5:
                    ups.append("x = 0")
                if rng.random() < 0.2:
                    if rng.random() < 0.5 and s not in receivers and j != spine[s]:
                        labels.append(("synchronisation", "bc?"))
                        receivers.add(s)
                    else:
                        labels.append(("synchronisation", "bc!"))
            labels.insert(0, ("guard", " && ".join(guards)))
            if ups:
                labels.append(("assignment", ", ".join(ups)))
            trans_by_src[s].append((j, (ids[s], ids[t], labels), escape_edge))
        trans = []
        for l in range(n_locs):
            # the escape edge of an invariant location goes last
            lst = sorted(trans_by_src[l], key=lambda e: (e[2], e[0]))
            trans.extend(e[1] for e in lst)
        init = ids[rng.randrange(n_locs)]
        d.template(f"C{c}", "clock x;", locs, init, trans)
    return Workload(f"random_{seed}", d.finish(), var_id=0, threshold=target - 1, horizon=horizon, runs=runs,
                    n_vars=2 + n_comps)


def batch_networks(count: int = 64, base_seed: int = 1000):
    """Uneven random networks: components log-uniform in [2, 512], 2..8
    locations, horizon U[50, 500], run budget log-uniform in [1e3, 1e6]."""
    out = []
    for i in range(count):
        rng = random.Random(base_seed + i)
        comps = int(round(math.exp(rng.uniform(math.log(2), math.log(512)))))
        locs = rng.randint(2, 8)
        edges = locs + rng.randint(0, locs)
        horizon = rng.randint(50, 500)
        budget = int(round(math.exp(rng.uniform(math.log(1e3), math.log(1e6)))))
        w = random_network(base_seed + i, n_comps=comps, n_locs=locs, n_edges=edges, horizon=horizon,
                           runs=budget)
        w.name = f"batch_{i}"
        out.append(w)
    return out


def expression_zoo(seed: int, full: bool = False) -> Workload:
    """A small random network that exercises the front end's expression
    language: integer, double and constant operands, + - * / (and with full:
    %, unary minus, sqrt(), random(), || and negated guards), comparisons and
    conjunctions in guards, conditional assignments c ? a : b, clock guards
    and invariants, exponential rates given as expressions, committed and
    urgent locations, branchpoints with probability weights, broadcast
    senders and receivers, local clocks and ints.  Every location lies on a
    cycle through the template, so it is reachable.  Many full models fall
    outside the subset the reference front end accepts; the front end must
    then reject them as the reference does.  Query Pr[<=50](<> v0 >= 4)."""
    rng = random.Random(seed)

    def operand(ints, dbls):
        r = rng.random()
        if r < 0.45:
            return rng.choice(ints)
        if r < 0.6 and dbls:
            return rng.choice(dbls)
        if r < 0.85:
            return str(rng.randint(0, 9))
        return f"{rng.randint(0, 9)}.{rng.randint(0, 99)}"

    def expr(depth, ints, dbls, cond_ok=False):
        if depth <= 0 or rng.random() < 0.3:
            return operand(ints, dbls)
        k = rng.random()
        if k < 0.55:
            ops = ["+", "-", "*", "/", "%"] if full else ["+", "-", "*", "/"]
            return f"({expr(depth - 1, ints, dbls)} {rng.choice(ops)} {expr(depth - 1, ints, dbls)})"
        if full and k < 0.65:
            return f"-{expr(depth - 1, ints, dbls)}"
        if full and k < 0.75:
            return f"sqrt({expr(depth - 1, ints, dbls)})"
        if full and k < 0.8:
            return f"random({rng.randint(1, 9)})"
        if cond_ok and k < 0.9:
            return f"{cond(depth - 1, ints, dbls)} ? {expr(depth - 1, ints, dbls)} : {expr(depth - 1, ints, dbls)}"
        return f"({expr(depth - 1, ints, dbls)})"

    def cond(depth, ints, dbls):
        op = rng.choice(["<", "<=", ">", ">=", "==", "!="])
        return f"{rng.choice(ints)} {op} {expr(max(0, depth - 1), ints, dbls)}"

    def guard(ints, dbls, clocks):
        parts = []
        for _ in range(rng.randint(1, 3)):
            if clocks and rng.random() < 0.4:
                parts.append(f"{rng.choice(clocks)} {rng.choice(['>=', '>', '<=', '<'])} {rng.randint(0, 9)}")
            else:
                parts.append(cond(2, ints, dbls))
        g = (rng.choice([" && ", " && ", " || "]) if full else " && ").join(parts)
        if full and rng.random() < 0.1:
            g = "!(" + g + ")"
        return g

    ints = [f"v{i}" for i in range(rng.randint(1, 4))]
    dbls = [f"d{i}" for i in range(rng.randint(0, 2))]
    consts = [f"K{i}" for i in range(rng.randint(0, 2))]
    decl = [f"int {v} = {rng.randint(0, 5)};" for v in ints]
    decl += [f"double {d} = {rng.randint(0, 5)}.{rng.randint(0, 9)};" for d in dbls]
    decl += [f"const int {c} = {rng.randint(1, 9)};" for c in consts]
    decl += ["broadcast chan b;"]
    parts = ['<?xml version="1.0" encoding="utf-8"?>', "<nta>", f"<declaration>{escape(chr(10).join(decl))}</declaration>"]
    counter = [0]

    def new_id():
        counter[0] += 1
        return f"id{counter[0]}"

    names = []
    for t in range(rng.randint(1, 4)):
        name = f"T{t}"
        clocks = ["x"] if rng.random() < 0.7 else []
        local = (["clock x;"] if clocks else []) + ([f"int w = {rng.randint(0, 3)};"] if rng.random() < 0.3 else [])
        lints = ints + consts + (["w"] if any(s.startswith("int w") for s in local) else [])
        n = rng.randint(2, 5)
        ids = [new_id() for _ in range(n)]
        parts += ["<template>", f"<name>{name}</name>", f"<declaration>{escape(chr(10).join(local))}</declaration>"]
        for i, lid in enumerate(ids):
            parts += [f'<location id="{lid}">', f"<name>L{i}</name>"]
            r = rng.random()
            if clocks and r < 0.25:
                parts.append(_label("invariant", f"x <= {rng.randint(2, 9)}"))
            elif r < 0.7:
                rate = expr(2, lints, dbls) if rng.random() < 0.4 else str(rng.randint(1, 5))
                parts.append(_label("exponentialrate", rate))
            if rng.random() < 0.1:
                parts.append("<committed/>")
            elif rng.random() < 0.1:
                parts.append("<urgent/>")
            parts.append("</location>")
        bp = new_id() if rng.random() < 0.4 else None
        if bp:
            parts.append(f'<branchpoint id="{bp}"/>')
        parts.append(f'<init ref="{ids[0]}"/>')
        for i in range(n):
            outs = rng.randint(1, 3)
            for o in range(outs):
                last = o == outs - 1  # the cycle edge i -> i + 1
                dst = ids[(i + 1) % n] if last else ids[rng.randrange(n)]
                if bp and o == 0 and not last and rng.random() < 0.5:
                    dst = bp
                parts += ["<transition>", f'<source ref="{ids[i]}"/>', f'<target ref="{dst}"/>']
                if rng.random() < 0.7:
                    parts.append(_label("guard", guard(lints, dbls, clocks)))
                if rng.random() < 0.2:
                    parts.append(_label("synchronisation", "b" + rng.choice(["!", "?"])))
                ups = [f"{rng.choice(ints + (['w'] if 'w' in lints else []) + dbls)} = "
                       f"{expr(3, lints, dbls, cond_ok=True)}" for _ in range(rng.randint(0, 3))]
                if clocks and rng.random() < 0.4:
                    ups.append("x = 0")
                if ups:
                    parts.append(_label("assignment", ", ".join(ups)))
                if rng.random() < 0.2:
                    parts.append(_label("probability", str(rng.randint(1, 5))))
                parts.append("</transition>")
        if bp:
            for _ in range(rng.randint(1, 3)):
                parts += ["<transition>", f'<source ref="{bp}"/>', f'<target ref="{ids[rng.randrange(n)]}"/>',
                          _label("probability", str(rng.randint(1, 5)))]
                if rng.random() < 0.5:
                    parts.append(_label("assignment", f"{rng.choice(ints)} = {expr(2, lints, dbls)}"))
                parts.append("</transition>")
        parts.append("</template>")
        names.append(name)
    parts += [f"<system>system {', '.join(names)};</system>", "</nta>"]
    return Workload(f"zoo{'_full' if full else ''}_{seed}", "\n".join(parts) + "\n", var_id=0, threshold=3,
                    horizon=50, runs=10_000)
