"""Editing the schedule fields of serialized IR text (the reference's
format, serialization.cpp:175-237: node lines n:op:inputs:vars:constraints:
sym_map:priority:order:reuse:loop_annotations:annotation), as the
reference's IR::set_order / annotate_loop would."""


def node_lines(text):
    lines = text.splitlines()
    return lines, [i for i, ln in enumerate(lines) if ln.startswith("n:")]


def get_order(text, node):
    lines, nl = node_lines(text)
    f = lines[nl[node]].split(":")
    order = [tuple(int(x) for x in e.split(";")) for e in f[7].split(",") if e]
    annots = f[9].split(",")[:len(order)]
    annots += [""] * (len(order) - len(annots))
    return order, annots


def set_order(text, node, order, annots=None):
    """order: [(var, size, tail), ...]; annots: one string per entry."""
    lines, nl = node_lines(text)
    f = lines[nl[node]].split(":")
    f[7] = "".join(f"{v};{s};{t}," for v, s, t in order)
    f[9] = "".join(f"{a}," for a in (annots or [""] * len(order)))
    lines[nl[node]] = ":".join(f)
    return "\n".join(lines) + "\n"


def nodes_with_loops(text):
    lines, nl = node_lines(text)
    return [k for k, i in enumerate(nl) if lines[i].split(":")[7]]
