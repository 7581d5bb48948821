"""Description text of a workloads.Netlist for the reference harness
(nsref_sim_run in oracle/ref_shim.cpp): the same device list, built through
the reference's typed Circuit API in the same order."""


def ref_desc(netlist, options=None) -> str:
    lines = [f"nodes {netlist.num_nodes}"]
    for name, (mtype, params) in getattr(netlist, "models", {}).items():
        level = int(params.get("LEVEL", 1))
        card = " ".join(f"{k.lower()}={float(v)!r}" for k, v in params.items() if k != "LEVEL")
        lines.append(f"MODEL .model {name} {mtype} (level={level} {card})")
    for d in netlist.devices:
        if d[0] == "M":
            lines.append(" ".join(["M"] + [repr(int(x)) for x in d[1:5]] +
                                  [d[5]] + [repr(float(x)) for x in d[6:]]))
            continue
        lines.append(" ".join([d[0]] + [repr(int(x)) for x in d[1:3]] +
                              [repr(float(x)) for x in d[3:]]))
    for k, v in (options or {}).items():
        lines.append(f"OPT {k} {float(v)!r}")  # plain float repr (not numpy's np.float64(...))
    return "\n".join(lines) + "\n"
