"""CPU restatement of the reference's GAR match C-ABI path — TEST INFRASTRUCTURE ONLY.

Imported only by tests/ as the checker of ``matrixgraph_gar_match``.  Pure
Python: meant for graphs of a few hundred edges.

Two modes share the input conventions and the output writer:

* ``mode="reference"`` follows the reference step by step:
  ``matrixgraph_gar_match`` (core/go_api/matrixgraph_go_api.cu:209-227) ->
  ``GARMatch::Run`` (core/task/gpu_task/gar_match.cu:193-240) ->
  ``GARMatchKernelWrapper::GARMatch``
  (core/task/gpu_task/kernel/kernel_gar_match.cu:365-709): per pattern edge
  the data-edge candidates that pass the vertex filters (LabelDegree,
  NeighborLabelCounter, KMinWiseIP; :49-214), then the edge-at-a-time
  frontier join (:299-363), then the pivot-grouped flattening (:640-700).
  The reference keeps at most ``match_capacity / n_nodes`` frontier rows per
  join step and drops the excess in atomic-arrival order
  (:527-531, :331-334), so its output is only determined when no step
  overflowed; ``truncated`` reports whether one did.
* ``mode="exact"``: every injective map of the pattern nodes that preserves
  node labels and maps each pattern edge onto a data edge with the same edge
  label, by backtracking; no filters, no frontier cap.  This is what the
  library computes.

Both return the outputs of the C entry point as a GarResult.  Where the
reference filters reject no vertex that an exact match uses and no step
overflowed, the two modes agree; ``filters_pruned`` reports whether they
rejected one.
"""
from __future__ import annotations

from dataclasses import dataclass, field

KMAX_VERTEX_ID = 0xFFFFFFFF      # kMaxVertexID, core/common/consts.h:15
HEAP_CAPACITY = 7                # kDefaultHeapCapacity, core/common/consts.h:47
# Label hash of the k-min-wise filter: HashTable, kernel/algorithms/hash.cuh:31-65
# (keys 0..15 mapped to a permutation of 0..15, every other key to 0).
_HASH_TABLE = (12, 3, 11, 9, 15, 2, 8, 4, 13, 10, 5, 7, 14, 6, 1, 0)


def _hash_table(key: int) -> int:
    return _HASH_TABLE[key] if 0 <= key < 16 else 0


def _u32(x: int) -> int:
    return x & 0xFFFFFFFF


class _Heap:
    """MinHeap of core/data_structures/heap.cuh:18-111, as written: the
    insertion step swaps with the parent at most once (the loop never moves
    its index), and the replacement step compares the left child with '>'
    and the right child with '<'."""

    def __init__(self):
        self.data = [0] * HEAP_CAPACITY
        self.offset = 0

    def insert(self, val: int) -> None:
        d = self.data
        if self.offset < HEAP_CAPACITY:
            d[self.offset] = val
            self.offset += 1
            i = self.offset - 1
            while i > 0:
                parent = (i - 1) // 2
                if d[i] > d[parent]:
                    d[i], d[parent] = d[parent], d[i]
                else:
                    break
        elif val < d[0]:
            d[0] = val
            self._heapify(0)

    def _heapify(self, i: int) -> None:
        d = self.data
        largest = i
        while True:
            left, right = 2 * i + 1, 2 * i + 2
            if left < self.offset and d[left] > d[largest]:
                largest = left
            if right < self.offset and d[right] < d[largest]:
                largest = right
            if largest == i:
                break
            d[i], d[largest] = d[largest], d[i]
            i = largest


def _bitmap_count(x: int) -> int:
    """MiniKernelBitmap::Count (core/data_structures/mini_kernel_bitmap.cuh:53-63)
    with its masks as written (bits 29-31 are not counted)."""
    x = _u32(x)
    x = (x & 0x55555555) + ((x >> 1) & 0x5555555)
    x = (x & 0x33333333) + ((x >> 2) & 0x3333333)
    x = (x & 0x0F0F0F0F) + ((x >> 4) & 0xF0F0F0F)
    x = (x & 0x00FF00FF) + ((x >> 8) & 0x0FF00FF)
    x = (x & 0x0000FFFF) + ((x >> 16) & 0x0000FFFF)
    return x


@dataclass
class GarGraph:
    """GARGraphArrays (core/data_structures/gar_graph_arrays.h): vertices by
    local index with instance ids and labels; directed edges by local index."""
    v_id: list | None
    v_label: list | None
    e_src: list
    e_dst: list
    e_label: list | None = None
    n_vertices: int | None = None

    def __post_init__(self):
        if self.n_vertices is None:
            self.n_vertices = len(self.v_label) if self.v_label is not None else 0


@dataclass
class GarPattern:
    """GARPatternArrays (core/data_structures/gar_pattern_arrays.h)."""
    node_label: list | None
    edge_src: list
    edge_dst: list
    edge_label: list | None = None
    n_nodes: int | None = None

    def __post_init__(self):
        if self.n_nodes is None:
            self.n_nodes = len(self.node_label) if self.node_label is not None else 0


@dataclass
class GarResult:
    rc: int = 0
    num_conditions: int = 0
    row_pivot_id: list = field(default_factory=list)
    row_cond_j: list = field(default_factory=list)
    row_pos: list = field(default_factory=list)
    row_offset: list = field(default_factory=list)
    row_count: list = field(default_factory=list)
    matched_v_ids: list = field(default_factory=list)
    truncated: bool = False
    filters_pruned: bool = False
    n_embeddings: int = 0          # distinct complete node maps

    @property
    def row_size(self) -> int:
        return len(self.row_pivot_id)

    @property
    def match_size(self) -> int:
        return len(self.matched_v_ids)


# ---- vertex filters (kernel_gar_match.cu:49-214) -------------------------------
def _p_degrees(p: GarPattern, u: int):
    po = sum(1 for e in range(len(p.edge_src)) if p.edge_src[e] == u)
    pi = sum(1 for e in range(len(p.edge_src)) if p.edge_dst[e] == u)
    return po, pi


def _g_degrees(g: GarGraph, v: int):
    go = sum(1 for s in g.e_src if s == v)
    gi = sum(1 for d in g.e_dst if d == v)
    return go, gi


def _label_degree(p, g, u, v) -> bool:
    if u < 0 or u >= p.n_nodes or v >= g.n_vertices:
        return False
    if p.node_label is None or g.v_label is None:
        return False
    if p.node_label[u] != g.v_label[v]:
        return False
    po, pi = _p_degrees(p, u)
    go, gi = _g_degrees(g, v)
    return go >= po and gi >= pi


def _p_nbr_labels(p, u):
    """Neighbour labels of pattern node u, one per incident edge (direction
    order of the reference loop: out-edge label first, then in-edge label)."""
    out = []
    for e in range(len(p.edge_src)):
        s, d = p.edge_src[e], p.edge_dst[e]
        if s == u and 0 <= d < p.n_nodes:
            out.append(_u32(p.node_label[d]) & 31)
        if d == u and 0 <= s < p.n_nodes:
            out.append(_u32(p.node_label[s]) & 31)
    return out


def _g_nbr_labels(g, v):
    out = []
    n = g.n_vertices
    for e in range(len(g.e_src)):
        s, d = g.e_src[e], g.e_dst[e]
        if s == v and d < n:
            out.append(_u32(g.v_label[d]) & 31)
        if d == v and s < n:
            out.append(_u32(g.v_label[s]) & 31)
    return out


def _nlc(p, g, u, v) -> bool:
    if u < 0 or u >= p.n_nodes or v >= g.n_vertices:
        return False
    if p.node_label is None or g.v_label is None:
        return False
    if p.node_label[u] != g.v_label[v]:
        return False
    ub = vb = 0
    for lab in _p_nbr_labels(p, u):
        ub |= 1 << lab
    for lab in _g_nbr_labels(g, v):
        vb |= 1 << lab
    return _bitmap_count(vb) >= _bitmap_count(ub)


def _kminwise(p, g, u, v) -> bool:
    if u < 0 or u >= p.n_nodes or v >= g.n_vertices:
        return False
    if p.node_label is None or g.v_label is None:
        return False
    if p.node_label[u] != g.v_label[v]:
        return False
    po, pi = _p_degrees(p, u)
    go, gi = _g_degrees(g, v)
    ub = vb = 0
    uh, vh = _Heap(), _Heap()
    for lab in _p_nbr_labels(p, u):
        ub |= 1 << lab
        uh.insert(_hash_table(lab))
    for lab in _g_nbr_labels(g, v):
        vb |= 1 << lab
        vh.insert(_hash_table(lab))
    ud, vd = list(uh.data), list(vh.data)
    for i in range(vh.offset):
        for j in range(uh.offset):
            if ud[j] == vd[i]:
                vd[i] = KMAX_VERTEX_ID
                ud[j] = KMAX_VERTEX_ID
                break
    min_v = KMAX_VERTEX_ID
    for i in range(vh.offset):
        min_v = min(min_v, vd[i])
    for j in range(uh.offset):
        if ud[j] < min_v:
            return False
    return _bitmap_count(vb) >= _bitmap_count(ub) and go >= po and gi >= pi


def _vertex_filter(p, g, u, v) -> bool:
    return _label_degree(p, g, u, v) and _nlc(p, g, u, v) and _kminwise(p, g, u, v)


# ---- candidates and join (kernel_gar_match.cu:262-363, :386-660) ----------------
def _edge_candidates(p, g, pe, filters=True):
    pu, pv = p.edge_src[pe], p.edge_dst[pe]
    plab = p.edge_label[pe] if p.edge_label is not None else 0
    n = g.n_vertices
    if filters:
        src_ok = {v: _vertex_filter(p, g, pu, v) for v in range(n)}
        dst_ok = {v: _vertex_filter(p, g, pv, v) for v in range(n)}
    out = []
    for ge in range(len(g.e_src)):
        if g.e_label is not None and g.e_label[ge] != plab:
            continue
        gs, gd = g.e_src[ge], g.e_dst[ge]
        if gs >= n or gd >= n or g.v_label is None:
            continue
        if g.v_label[gs] != p.node_label[pu] or g.v_label[gd] != p.node_label[pv]:
            continue
        if filters and (not src_ok[gs] or not dst_ok[gd]):
            continue
        out.append((gs, gd))
    return out


def _join(p, cands, max_embeddings):
    """Frontier join; returns (complete embeddings with multiplicity, truncated)."""
    k = p.n_nodes
    truncated = False
    u0, v0 = p.edge_src[0], p.edge_dst[0]
    front = []
    for gs, gd in cands[0]:
        if u0 == v0 and gs != gd:
            continue
        if u0 != v0 and gs == gd:
            continue
        row = [-1] * k
        row[u0], row[v0] = gs, gd
        front.append(row)
    if len(front) > max_embeddings:
        truncated = True
    for pe in range(1, len(p.edge_src)):
        if not front:
            break
        pu, pv = p.edge_src[pe], p.edge_dst[pe]
        nxt = []
        for row in front:
            for gs, gd in cands[pe]:
                if pu == pv and gs != gd:
                    continue
                if pu != pv and gs == gd:
                    continue
                au, av = row[pu], row[pv]
                if au >= 0 and au != gs:
                    continue
                if av >= 0 and av != gd:
                    continue
                if au < 0 and gs in row:
                    continue
                if av < 0 and gd in row:
                    continue
                r = list(row)
                r[pu], r[pv] = gs, gd
                nxt.append(r)
        if len(nxt) > max_embeddings:
            truncated = True
        front = nxt
    return [r for r in front if all(x >= 0 for x in r)], truncated


def _exact_embeddings(p, g):
    """Backtracking over pattern nodes 0..k-1 (node label, edge label and
    direction preserving, injective)."""
    k, n = p.n_nodes, g.n_vertices
    has = set()
    for ge in range(len(g.e_src)):
        gs, gd = g.e_src[ge], g.e_dst[ge]
        if gs < n and gd < n:
            has.add((gs, gd, g.e_label[ge] if g.e_label is not None else None))
    pedges = []
    for pe in range(len(p.edge_src)):
        pl = p.edge_label[pe] if p.edge_label is not None else 0
        pedges.append((p.edge_src[pe], p.edge_dst[pe], None if g.e_label is None else pl))
    by_label = {}
    for v in range(n):
        by_label.setdefault(g.v_label[v], []).append(v)
    out = []
    f = [-1] * k

    def ok(u):
        for s, d, lab in pedges:
            if max(s, d) <= u and (s == u or d == u):
                if (f[s], f[d], lab) not in has:
                    return False
        return True

    def rec(u):
        if u == k:
            out.append(list(f))
            return
        for v in by_label.get(p.node_label[u], []):
            if v in f[:u]:
                continue
            f[u] = v
            if ok(u):
                rec(u + 1)
            f[u] = -1

    rec(0)
    return out


def _flatten(g, embeddings, n_nodes, row_capacity, match_capacity, res: GarResult):
    """Pivot-grouped output (kernel_gar_match.cu:640-700): groups by the data
    vertex of pattern node 0 in local-index order; per pattern position the
    sorted distinct instance ids; rows and ids cut at the capacities."""
    def inst(v):
        if g.v_id is not None and v < g.n_vertices:
            return g.v_id[v]
        return v

    embeddings = sorted(embeddings, key=lambda e: e[0])
    row_size = match_size = 0
    i = 0
    stop = False
    while i < len(embeddings) and not stop:
        pivot = embeddings[i][0]
        j = i
        while j < len(embeddings) and embeddings[j][0] == pivot:
            j += 1
        for pos in range(n_nodes):
            vals = sorted(set(inst(embeddings[t][pos]) for t in range(i, j)))
            if row_size >= row_capacity:
                break
            offset = match_size
            write_n = len(vals)
            if offset + write_n > match_capacity:
                write_n = max(0, match_capacity - offset)
            res.row_pivot_id.append(inst(pivot))
            res.row_cond_j.append(pos)
            res.row_pos.append(pos)
            res.row_offset.append(offset)
            res.row_count.append(write_n)
            res.matched_v_ids.extend(vals[:write_n])
            match_size += write_n
            row_size += 1
            if row_size >= row_capacity or match_size >= match_capacity:
                break
        if row_size >= row_capacity or match_size >= match_capacity:
            stop = True
        i = j
    res.num_conditions = n_nodes


def gar_match(g: GarGraph, p: GarPattern, row_capacity: int, match_capacity: int,
              mode: str = "exact", check_filters: bool | None = None) -> GarResult:
    """Outputs of the C entry point for one (graph, pattern) pair.
    ``check_filters`` (default: reference mode only) evaluates the reference
    vertex filters to set ``filters_pruned``; they scan every data edge per
    vertex, so keep it off for graphs beyond a few hundred edges."""
    if check_filters is None:
        check_filters = mode == "reference"
    res = GarResult(num_conditions=1)
    k = p.n_nodes
    ready = (len(g.e_src) > 0 and len(p.edge_src) > 0 and p.node_label is not None)
    if k <= 0 or len(p.edge_src) <= 0:
        return res
    valid = all(0 <= p.edge_src[e] < k and 0 <= p.edge_dst[e] < k
                for e in range(len(p.edge_src)))
    if not ready or not valid or g.v_label is None:
        return res
    covered = set(p.edge_src) | set(p.edge_dst)
    exact = _exact_embeddings(p, g) if len(covered) == k else []
    if check_filters or mode == "reference":
        ref_cands = [_edge_candidates(p, g, pe, filters=True) for pe in range(len(p.edge_src))]
        # Did the reference filters drop a candidate edge that an exact match uses?
        ref_sets = [set(c) for c in ref_cands]
        res.filters_pruned = any((e[p.edge_src[pe]], e[p.edge_dst[pe]]) not in ref_sets[pe]
                                 for e in exact for pe in range(len(p.edge_src)))
    if mode == "reference":
        if any(len(c) == 0 for c in ref_cands):
            return res
        max_emb = max(1, int(match_capacity / max(1, k)))
        embs, res.truncated = _join(p, ref_cands, max_emb)
    elif mode == "exact":
        embs = exact
    else:
        raise ValueError(mode)
    distinct = {tuple(e) for e in embs}
    res.n_embeddings = len(distinct)
    if not embs:
        return res
    _flatten(g, [list(e) for e in embs], k, row_capacity, match_capacity, res)
    return res
