"""CPU restatement of the reference's generic path -- TEST INFRASTRUCTURE ONLY.

Nothing in the product imports this module: it is the checker of the GPU
generic path (sbdgpu_genop_*) in tests/.  It restates, in plain Python and
numpy, for small cases:

* NormalOrdering of a ProductOp and of a GeneralOp, and Simplify
  (r-ccs-cms/sbd include/sbd/basic/out_of_place_func/arithmetic.h:43-337):
  an annihilator directly followed by a creator is rewritten as
  c_x c+_y = delta_xy + s c+_y c_x (s = -1 with sign, +1 without), the
  creators are then sorted by ascending site and the annihilators by
  descending site (s per transposition), products that repeat a site among
  their creators or among their annihilators are dropped, equal products are
  summed, sums of magnitude <= 1e-8 dropped, and each product is filed as
  diagonal or off-diagonal by ProductOp::check_diagonal (generalop.h:288-319);
* GeneralOp_From_FCIDump (stdmodel.h:13-98): the quantum-chemistry
  Hamiltonian on 2L sites (alpha orbital p at site p, beta at site p + L);
* mult (mult.h:118-291 at one rank): the diagonal list adds coef * C_i when
  the sites of a term's first n_dag operators are occupied; an off-diagonal
  term annihilates the sites of its first n_dag operators from the bra state
  in turn and creates the rest, each operator contributing (-1)^(occupied
  sites below it) with sign (framework/bit_manipulation.h:943-962), and adds
  coef * sign * C_j for the basis state j reached.  The reference finds j with
  Basis::IndexSearch (basis.h:317-322), whose bisection is bounded by the
  target's word count instead of the basis size, so it finds (or, with the
  bound it gets, loops on) only the first states; this restatement searches
  the whole basis, as the search is evidently meant to;
* Lanczos (lanczos.h:176-310), with its second pass for the Ritz vector;
* an independent dense matrix of a product of field operators in the
  Jordan-Wigner convention |x> = prod_{q in x, ascending} c+_q |0>, which pins
  the sign rule above.
"""
from __future__ import annotations

import numpy as np

# ---------------------------------------------------------------- algebra


def _check_diagonal(ops):
    """generalop.h:288-319: as many creators as annihilators, and every
    creator's site also annihilated by another operator of the product."""
    nc = sum(1 for d, _ in ops if d)
    if nc != len(ops) - nc:
        return False
    for i, (d, q) in enumerate(ops):
        if d and not any(j != i and (not dj and qj == q) for j, (dj, qj) in enumerate(ops)):
            return False
    return True


def _inversions(seq, key):
    n = 0
    for i in range(len(seq)):
        for j in range(i + 1, len(seq)):
            if key(seq[j]) < key(seq[i]):
                n += 1
    return n


def normal_order_product(ops, sign=True):
    """One product (list of (dag, site)) -> (diag, off) lists of (coef, ops)."""
    s = -1.0 if sign else 1.0
    work = [(1.0, list(ops))]
    ordered = []
    while work:
        c, o = work.pop(0)
        k = next((i for i in range(len(o) - 1) if not o[i][0] and o[i + 1][0]), None)
        if k is None:
            ordered.append((c, o))
            continue
        work.append((c * s, o[:k] + [o[k + 1], o[k]] + o[k + 2:]))
        if o[k][1] == o[k + 1][1]:
            work.append((c, o[:k] + o[k + 2:]))
    sums = {}
    order = []
    for c, o in ordered:
        cr = [x for x in o if x[0]]
        an = [x for x in o if not x[0]]
        if len({q for _, q in cr}) < len(cr) or len({q for _, q in an}) < len(an):
            continue
        if sign:
            c *= (-1.0) ** (_inversions(cr, lambda x: x[1]) + _inversions(an, lambda x: -x[1]))
        key = tuple(sorted(cr, key=lambda x: x[1]) + sorted(an, key=lambda x: -x[1]))
        if key not in sums:
            order.append(key)
            sums[key] = 0.0
        sums[key] += c
    diag, off = [], []
    for key in order:
        v = sums[key]
        if abs(v) > 1e-8:
            (diag if _check_diagonal(key) else off).append((v, list(key)))
    return diag, off


def normal_order(G, sign=True):
    """arithmetic.h:247-287: every term of both lists, in turn, scaled by its
    coefficient; no summation across terms."""
    diag, off = [], []
    for lst in (G[0], G[1]):
        for c, ops in lst:
            d, o = normal_order_product(ops, sign)
            diag += [(c * v, p) for v, p in d]
            off += [(c * v, p) for v, p in o]
    return diag, off


def simplify(G):
    """arithmetic.h:288-337: equal products summed within each list."""
    out = []
    for lst in G:
        sums, order = {}, []
        for c, ops in lst:
            key = tuple(ops)
            if key not in sums:
                order.append(key)
                sums[key] = 0.0
            sums[key] += c
        out.append([(sums[k], list(k)) for k in order if abs(sums[k]) > 1e-8])
    return out[0], out[1]


def from_fcidump(L, integrals):
    """stdmodel.h:13-98: integrals in file order as (value, i, j, k, l), 1-based."""
    H = ([], [])
    for value, i, j, k, l in integrals:
        if i == 0 and j == 0 and k == 0 and l == 0:
            H[0].append((value, []))
        elif k == 0 and l == 0:
            idx = sorted({(i, j), (j, i)})
            T = ([], [])
            for p0, p1 in idx:
                T[1].append((value, [(True, p0 - 1), (False, p1 - 1)]))
                T[1].append((value, [(True, p0 - 1 + L), (False, p1 - 1 + L)]))
            T = simplify(normal_order(T, True))
            H[0].extend(T[0])
            H[1].extend(T[1])
        else:
            idx = sorted({(i, j, k, l), (j, i, k, l), (i, j, l, k), (j, i, l, k),
                          (k, l, i, j), (k, l, j, i), (l, k, i, j), (l, k, j, i)})
            V = ([], [])
            for p in idx:
                for sa, sb in ((0, 0), (0, L), (L, 0), (L, L)):
                    V[1].append((0.5 * value, [(True, p[0] - 1 + sa), (True, p[2] - 1 + sb),
                                               (False, p[3] - 1 + sb), (False, p[1] - 1 + sa)]))
            V = simplify(normal_order(V, True))
            H[0].extend(V[0])
            H[1].extend(V[1])
    return H


# ---------------------------------------------------------------- mult



def _state_int(states, i):
    row = np.atleast_1d(states[i])
    v = 0
    for w, word in enumerate(row):
        v |= int(word) << (64 * w)
    return v


def mult(states, H, C, W=None, sign=True):
    """W + H C on the basis `states` ([n] or [n, nwords] uint64)."""
    st = np.asarray(states, dtype=np.uint64)
    n = st.shape[0]
    ints = [_state_int(st, i) for i in range(n)]
    index = {v: i for i, v in enumerate(ints)}
    out = np.zeros(n) if W is None else np.array(W, dtype=np.float64)
    diag, off = H
    for i, v in enumerate(ints):
        acc = out[i]
        for c, ops in diag:
            nd = sum(1 for d, _ in ops if d)
            if all((v >> q) & 1 for _, q in ops[:nd]):
                acc += c * C[i]
        for c, ops in off:
            nd = sum(1 for d, _ in ops if d)
            w, s, ok = v, 1, True
            for k, (_, q) in enumerate(ops):
                if k < nd:
                    if not (w >> q) & 1:
                        ok = False
                        break
                    w &= ~(1 << q)
                else:
                    if (w >> q) & 1:
                        ok = False
                        break
                    w |= 1 << q
                if sign and bin(w & ((1 << q) - 1)).count("1") & 1:
                    s = -s
            if not ok:
                continue
            j = index.get(w)
            if j is not None:
                acc += c * s * C[j]
        out[i] = acc
    return out


def dense(states, H, sign=True):
    """<i|H|j> built column by column from mult (small bases only)."""
    n = np.asarray(states).shape[0]
    M = np.zeros((n, n))
    for j in range(n):
        e = np.zeros(n)
        e[j] = 1.0
        M[:, j] = mult(states, H, e, sign=sign)
    return M


def jordan_wigner(states, terms, nsites):
    """Independent dense matrix of sum_t coef_t * prod(ops_t) (ops applied
    right to left to the ket) in the convention |x> = prod_{q in x,
    ascending} c+_q |0>: c+_q / c_q pick up (-1)^(occupied sites below q)."""
    st = np.asarray(states, dtype=np.uint64)
    n = st.shape[0]
    ints = [_state_int(st, i) for i in range(n)]
    index = {v: i for i, v in enumerate(ints)}
    M = np.zeros((n, n))
    for j, x in enumerate(ints):
        for c, ops in terms:
            w, s = x, 1
            for d, q in reversed(ops):
                occ = (w >> q) & 1
                if d == bool(occ):
                    s = 0
                    break
                if bin(w & ((1 << q) - 1)).count("1") & 1:
                    s = -s
                w ^= 1 << q
            if s and w in index:
                M[index[w], j] += c * s
    return M


# ---------------------------------------------------------------- solvers


def lanczos(states, H, W, max_it, eps, sign=True):
    """lanczos.h:176-310 on CPU: (lowest Ritz value, Ritz vector, steps)."""
    W = np.array(W, dtype=np.float64)
    C0 = W.copy()
    C1 = np.zeros_like(W)
    lda = max_it
    A = np.zeros((lda, lda))
    e_old = 1.0e8
    it_stop = 0
    steps = 0
    E = U = None
    for it in range(max_it):
        steps += 1
        C1 = mult(states, H, C0, C1, sign)
        aii = float(C0 @ C1)
        A[it, it] = aii
        E, U = np.linalg.eigh(A[:steps, :steps])
        if abs(E[0] - e_old) < eps or it + 1 == max_it:
            it_stop = it
            break
        e_old = E[0]
        C1 -= aii * C0
        b = float(np.linalg.norm(C1))
        C1 /= b
        A[it, it + 1] = A[it + 1, it] = b
        if abs(b) < eps:
            it_stop = it
            break
        C0, C1 = C1.copy(), -b * C0
    u = U[:, 0]
    C0 = W.copy()
    C1 = np.zeros_like(W)
    W = W * u[0]
    for it in range(it_stop):
        C1 = mult(states, H, C0, C1, sign)
        C1 -= A[it, it] * C0
        b = float(np.linalg.norm(C1))
        C1 /= b
        W += u[it + 1] * C1
        C0, C1 = C1.copy(), -b * C0
    return float(E[0]), W, steps


def read_fcidump(path):
    """(norb, nelec, integrals in file order as (value, i, j, k, l))."""
    header, ints = [], []
    with open(path) as f:
        in_header = True
        for line in f:
            if in_header:
                header.append(line)
                if "&END" in line.upper() or line.strip() == "/":
                    in_header = False
                continue
            parts = line.split()
            if len(parts) == 5:
                ints.append((float(parts[0]), *(int(x) for x in parts[1:])))
    text = " ".join(header).replace(",", " ").replace("=", " = ")
    tok = text.split()
    norb = int(tok[tok.index("NORB") + 2]) if "NORB" in tok else None
    nelec = int(tok[tok.index("NELEC") + 2]) if "NELEC" in tok else None
    return norb, nelec, ints


def _targets(v, ops, sign):
    """The state reached from bra v by one off-diagonal term (mult.h:213-240)
    and its sign, or None."""
    nd = sum(1 for d, _ in ops if d)
    w, s = v, 1
    for k, (_, q) in enumerate(ops):
        if k < nd:
            if not (w >> q) & 1:
                return None
            w &= ~(1 << q)
        else:
            if (w >> q) & 1:
                return None
            w |= 1 << q
        if sign and bin(w & ((1 << q) - 1)).count("1") & 1:
            s = -s
    return w, s


def ham_square(states, H, W, sign=True):
    """MeasHamSquare (expand.h:10-215): every basis state weighted by the
    diagonal list, every off-diagonal target weighted coef * sign * W_i, equal
    configurations summed, then the sum of squares."""
    st = np.asarray(states, dtype=np.uint64)
    ints = [_state_int(st, i) for i in range(st.shape[0])]
    diag, off = H
    acc = {}
    for i, v in enumerate(ints):
        val = 0.0
        for c, ops in diag:
            nd = sum(1 for d, _ in ops if d)
            if all((v >> q) & 1 for _, q in ops[:nd]):
                val += c * W[i]
        acc[v] = acc.get(v, 0.0) + val
        for c, ops in off:
            t = _targets(v, ops, sign)
            if t is not None:
                acc[t[0]] = acc.get(t[0], 0.0) + c * t[1] * W[i]
    return float(sum(x * x for x in acc.values()))


def expand(states, H, W, eps_hb, sign=True):
    """ExpandBasis (expand.h:217-366): the basis plus every off-diagonal
    target with |coef * sign * W_i| > eps_hb, sorted ascending as integers."""
    st = np.asarray(states, dtype=np.uint64)
    ints = [_state_int(st, i) for i in range(st.shape[0])]
    out = set(ints)
    for i, v in enumerate(ints):
        for c, ops in H[1]:
            t = _targets(v, ops, sign)
            if t is not None and abs(c * t[1] * W[i]) > eps_hb:
                out.add(t[0])
    return sorted(out)
