"""Counting the kernels a piece of work launches.

The work is captured once into a CUDA graph on torch's current device (the
capture records the launches without running them), and the graph's kernel
nodes are listed by function name through the CUDA driver.  The graph a
benchmark replays can be inspected the same way.
"""
import collections

import torch

PREFIX = "gprtcu"  # every kernel of libgprtcu.so lives in namespace gprtcu


def _check(res, what):
    err = res[0]
    if int(err) != 0:
        raise RuntimeError("%s failed: %s" % (what, err))
    return res[1:] if len(res) > 2 else res[1]


def _node_name(drv, node):
    params = _check(drv.cuGraphKernelNodeGetParams(node), "cuGraphKernelNodeGetParams")
    func = getattr(params, "func", None)
    if func is not None and int(func) != 0:
        name = _check(drv.cuFuncGetName(func), "cuFuncGetName")
    else:
        name = _check(drv.cuKernelGetName(params.kern), "cuKernelGetName")
    return name.decode() if isinstance(name, bytes) else str(name)


def graph_kernels(graph):
    """Kernel nodes of a torch.cuda.CUDAGraph made with keep_graph=True:
    Counter of mangled kernel names."""
    from cuda.bindings import driver as drv
    raw = drv.CUgraph(graph.raw_cuda_graph())
    _, count = _check(drv.cuGraphGetNodes(raw, 0), "cuGraphGetNodes")
    nodes, _ = _check(drv.cuGraphGetNodes(raw, count), "cuGraphGetNodes")
    names = collections.Counter()
    for node in nodes[:count]:
        kind = _check(drv.cuGraphNodeGetType(node), "cuGraphNodeGetType")
        if kind == drv.CUgraphNodeType.CU_GRAPH_NODE_TYPE_KERNEL:
            names[_node_name(drv, node)] += 1
    return names


def count_kernels(fn):
    """Kernels fn() launches (captured, not run).  Returns (ours, others):
    the number of this library's kernels and a Counter of any other kernels."""
    g = torch.cuda.CUDAGraph(keep_graph=True)
    with torch.cuda.graph(g):
        fn()
    names = graph_kernels(g)
    del g
    ours = sum(c for n, c in names.items() if PREFIX in n)
    others = collections.Counter({n: c for n, c in names.items() if PREFIX not in n})
    return ours, others

