"""One grid split into x slabs over ranks: the pipelined step.

The reference splits the x planes over MPI ranks (BioFVM_parallel.cpp:108-144)
and solves the x lines, which cross the ranks, with a pipelined exchange of
boundary planes (BioFVM_parallel.cpp:948-1255; the sends and receives at
:832-873): rank r's forward elimination of a block of lines starts from the
last forward values rank r-1 sends for them, and its back substitution from
the first back-substituted values rank r+1 sends. Blocks of lines keep every
rank busy while the others work on other blocks.

Here each rank holds a ``SlabEnv`` and four planes of ``slab.lines`` doubles
on its device: prev_in, prev_out, next_in, next_out. ``schedule`` lists one
rank's step as operations; ``step`` runs them with a transport the caller
supplies (bench.py and the tests wrap torch.distributed: NCCL between GPUs,
gloo between CPU processes), and ``emulate_step`` runs every rank's list in
one process, rank after rank, with plane copies standing in for the messages.

A ``planes`` object gives ptr(name) (the plane's device address) and, for
emulate_step, copy_from(name, src_planes, src_name, line0, line1), which must
return once the copy is complete. A transport gives send(name, line0, line1,
peer) and recv(name, line0, line1, peer) for the lines [line0, line1) of the
named plane, ordered with the slab env's stream.
"""
from __future__ import annotations

PLANES = ("prev_in", "prev_out", "next_in", "next_out")


def line_ranges(lines: int, blocks: int):
    """[line0, line1) of `blocks` near-equal blocks of the slab's lines."""
    blocks = max(1, min(blocks, lines))
    edges = [lines * b // blocks for b in range(blocks + 1)]
    return [(edges[b], edges[b + 1]) for b in range(blocks) if edges[b + 1] > edges[b]]


def schedule(rank: int, world: int, lines: int, blocks: int = 4):
    """One rank's step: per block of lines, receive prev_in, forward half, send
    prev_out; then per block, receive next_in, backward half, send next_out;
    then the slab's own y and z sweeps. Receives name the receiving plane,
    sends the sending one."""
    ops = []
    ranges = line_ranges(lines, blocks)
    for l0, l1 in ranges:
        if rank > 0:
            ops.append(("recv", "prev_in", l0, l1, rank - 1))
        ops.append(("forward", l0, l1))
        if rank < world - 1:
            ops.append(("send", "prev_out", l0, l1, rank + 1))
    for l0, l1 in ranges:
        if rank < world - 1:
            ops.append(("recv", "next_in", l0, l1, rank + 1))
        ops.append(("backward", l0, l1))
        if rank > 0:
            ops.append(("send", "next_out", l0, l1, rank - 1))
    ops.append(("yz",))
    return ops


def run_op(slab, dt, op, planes, transport=None):
    kind = op[0]
    if kind == "forward":
        slab.x_forward(dt, 0 if slab.first else planes.ptr("prev_in"), 0 if slab.last else planes.ptr("prev_out"),
                       op[1], op[2])
    elif kind == "backward":
        slab.x_backward(dt, 0 if slab.last else planes.ptr("next_in"), 0 if slab.first else planes.ptr("next_out"),
                        op[1], op[2])
    elif kind == "yz":
        slab.yz(dt)
    elif kind == "send":
        transport.send(op[1], op[2], op[3], op[4])
    elif kind == "recv":
        transport.recv(op[1], op[2], op[3], op[4])
    else:
        raise ValueError(f"unknown operation {kind!r}")


def step(slab, dt, rank: int, world: int, planes, transport, blocks: int = 4):
    """One LOD diffusion step of this rank's slab; every rank calls it."""
    for op in schedule(rank, world, slab.lines, blocks):
        run_op(slab, dt, op, planes, transport)


def emulate_step(slabs, dt, planes, blocks: int = 4):
    """Every rank's step in one process (all slabs on one device): each rank
    runs its operations in order until a receive whose message has not been
    sent; a send waits for the sender's work, then copies the lines into the
    receiver's plane. Ranks never wait inside a kernel: the host orders them."""
    R = len(slabs)
    ops = [schedule(r, R, slabs[r].lines, blocks) for r in range(R)]
    pos = [0] * R
    delivered = set()
    moved = True
    while moved:
        moved = False
        for r in range(R):
            while pos[r] < len(ops[r]):
                op = ops[r][pos[r]]
                if op[0] == "recv":
                    if (op[4], r, op[1], op[2], op[3]) not in delivered:
                        break
                elif op[0] == "send":
                    peer = op[4]
                    dst = "prev_in" if op[1] == "prev_out" else "next_in"
                    slabs[r].synchronize()
                    planes[peer].copy_from(dst, planes[r], op[1], op[2], op[3])
                    delivered.add((r, peer, dst, op[2], op[3]))
                else:
                    run_op(slabs[r], dt, op, planes[r])
                pos[r] += 1
                moved = True
    if any(pos[r] != len(ops[r]) for r in range(R)):
        raise RuntimeError("slab schedule stalled: a receive has no matching send")


def split_planes(nx_global: int, ranks: int):
    """(x0, nx_local) per rank: near-equal slabs covering every plane (the
    reference's x_nodes/dims[1] drops the remainder, BioFVM_parallel.cpp:108;
    here the first nx_global % ranks slabs take one plane more)."""
    if ranks < 1 or ranks > nx_global:
        raise ValueError("need 1 <= ranks <= nx_global")
    base, extra = divmod(nx_global, ranks)
    out, x0 = [], 0
    for r in range(ranks):
        n = base + (1 if r < extra else 0)
        out.append((x0, n))
        x0 += n
    return out
