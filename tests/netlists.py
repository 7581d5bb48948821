"""Description text of a workloads.Netlist for the reference harness
(nsref_sim_run in oracle/ref_shim.cpp): the same device list, built through
the reference's typed Circuit API in the same order."""


def ref_desc(netlist, options=None) -> str:
    lines = [f"nodes {netlist.num_nodes}"]
    for d in netlist.devices:
        lines.append(" ".join([d[0]] + [repr(int(x)) for x in d[1:3]] +
                              [repr(float(x)) for x in d[3:]]))
    for k, v in (options or {}).items():
        lines.append(f"OPT {k} {v!r}")
    return "\n".join(lines) + "\n"
