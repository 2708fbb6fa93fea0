"""Assignment of independent MCTDHB jobs to GPUs by HBM footprint.

The reference integrates one system per process (its globals, driver.c:15-19,
make it single-instance); independent systems shard with no exchange at
all.  Every rank runs the same deterministic assignment on the same job
list (sizes and seeds known to all), keeps its own share and never talks to
the other ranks in the data path.

`by_footprint` is the longest-processing-time rule: jobs in decreasing
footprint, each to the rank with the smallest total so far (ties: the
lowest rank).  Every job lands on exactly one rank, and the largest rank
total is at most the mean plus the largest single job (Graham's bound for
list scheduling), so per-rank arenas can be sized as mean + max.

`stream_by_footprint` assigns an arrival stream in arrival order: each job
goes to the rank with the least footprint admitted so far (the rank that
will have the most room), the same on every rank.
"""


def by_footprint(sizes, nranks):
    """list of job indices per rank, balancing sum(sizes) per rank"""
    if nranks < 1:
        raise ValueError("need at least one rank")
    load = [0] * nranks
    share = [[] for _ in range(nranks)]
    for i in sorted(range(len(sizes)), key=lambda k: (-sizes[k], k)):
        r = min(range(nranks), key=lambda q: (load[q], q))
        share[r].append(i)
        load[r] += sizes[i]
    for s in share:
        s.sort()
    return share


def stream_by_footprint(sizes, nranks):
    """rank of every job of an arrival stream (in arrival order)"""
    if nranks < 1:
        raise ValueError("need at least one rank")
    load = [0] * nranks
    out = []
    for b in sizes:
        r = min(range(nranks), key=lambda q: (load[q], q))
        out.append(r)
        load[r] += b
    return out


def loads(sizes, share):
    return [sum(sizes[i] for i in s) for s in share]
