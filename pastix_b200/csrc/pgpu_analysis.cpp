// Host analysis for grid problems: the reference's ordering, symbolic
// factorization, reordering and blend splitting, restated so that the GPU
// layer can run standalone.  The output is exactly the SolverMatrix and
// ordering the reference's analysis produces for the same grid (checked
// against the reference in tests/test_analysis.py):
//
//   1. pastixOrderGrid            order/order_grids.c:303  (nested dissection
//                                 of the nx x ny x nz grid, supernodes + tree)
//   2. orderApplyLevelOrder       order/order_apply_level_order.c (autolevel
//                                 2D-first breadth-first renumbering)
//   3. pastixSymbolFaxDirect      symbol/symbol_fax.c (block structure of L)
//   4. pastixSymbolReordering     symbol/symbol_reordering.c (per-supernode
//                                 pseudo-TSP on row contribution sets) and a
//                                 second symbolic factorization
//   5. splitSymbol                blend/splitsymbol.c + blend/extracblk.c
//                                 (split supernodes wider than MAX_BLOCKSIZE)
//   6. solverMatrixGen            blend/solver_matrix_gen.c (cblk/blok/browtab
//                                 tables of a single process)
#include "pastix_gpu.h"

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <memory>
#include <vector>

namespace {

using I = int64_t;
using VI = std::vector<I>;

struct Ordering {
    I n = 0, cblknbr = 0;
    VI permtab, peritab, rangtab, treetab;
};

struct Symbol {
    I cblknbr = 0, bloknbr = 0, nodenbr = 0;
    VI fcol, lcol, bloknum;            // cblk (bloknum has cblknbr+1 entries)
    VI frow, lrow, lcblk, fcblk;       // blok
    VI brownum, browtab;               // blocks facing each cblk (no diagonal)

    void build_rowtab() {
        brownum.assign(cblknbr + 1, 0);
        for (I b = 0; b < bloknbr; b++)
            if (fcblk[b] != lcblk[b]) brownum[fcblk[b] + 1]++;
        for (I c = 0; c < cblknbr; c++) brownum[c + 1] += brownum[c];
        browtab.assign(brownum[cblknbr], 0);
        VI pos(brownum.begin(), brownum.end() - 1);
        for (I c = 0; c < cblknbr; c++)
            for (I b = bloknum[c] + 1; b < bloknum[c + 1]; b++) browtab[pos[fcblk[b]]++] = b;
    }
};

// ---------------------------------------------------------------- step 1 --
// Recursive nested dissection of a box: separators numbered from the top of
// the remaining range downwards, leaves (< 15 vertices) numbered in place.
struct GridND {
    I ldx, ldy;
    VI &perm, &rang, &depth;
    I cblknbr = 0, next = 0, slot = 0;

    GridND(I lx, I ly, VI &p, VI &r, VI &d) : ldx(lx), ldy(ly), perm(p), rang(r), depth(d) {}

    void plane(I base, I a0, I a1, I b0, I b1, I sa, I sb) {
        for (I i = 0; i < a1 - a0; i++)
            for (I j = 0; j < b1 - b0; j++) perm[base + (a0 + i) * sa + (b0 + j) * sb] = next--;
    }

    void box(I x0, I x1, I y0, I y1, I z0, I z1, I lvl) {
        const I nx = x1 - x0, ny = y1 - y0, nz = z1 - z0;
        cblknbr++;
        depth[slot] = lvl;
        rang[slot] = next;
        slot++;
        if (nx * ny * nz < 15) {
            I cur = 0;
            for (I i = x0; i < x1; i++)
                for (I j = y0; j < y1; j++)
                    for (I k = z0; k < z1; k++) perm[i + ldx * j + ldx * ldy * k] = next - cur++;
            next -= cur;
            return;
        }
        int dir = (ny > nx) ? 1 : 0;
        if (nz > nx && nz > ny) dir = 2;
        if (dir == 0) {
            plane(x0 + nx / 2, y0, y1, z0, z1, ldx, ldx * ldy);
            box(x0, x0 + nx / 2, y0, y1, z0, z1, lvl + 1);
            box(x0 + nx / 2 + 1, x1, y0, y1, z0, z1, lvl + 1);
        } else if (dir == 1) {
            plane(ldx * (y0 + ny / 2), x0, x1, z0, z1, 1, ldx * ldy);
            box(x0, x1, y0, y0 + ny / 2, z0, z1, lvl + 1);
            box(x0, x1, y0 + ny / 2 + 1, y1, z0, z1, lvl + 1);
        } else {
            plane(ldx * ldy * (z0 + nz / 2), x0, x1, y0, y1, 1, ldx);
            box(x0, x1, y0, y1, z0, z0 + nz / 2, lvl + 1);
            box(x0, x1, y0, y1, z0 + nz / 2 + 1, z1, lvl + 1);
        }
    }
};

void order_grid(I nx, I ny, I nz, Ordering &o) {
    const I n = nx * ny * nz;
    o.n = n;
    o.permtab.assign(n, 0);
    VI rang(n + 1, 0), depth(n, 0);
    GridND nd(nx, ny, o.permtab, rang, depth);
    nd.next = n - 1;
    nd.box(0, nx, 0, ny, 0, nz, 1);
    const I cn = nd.cblknbr;
    o.cblknbr = cn;
    o.peritab.assign(n, 0);
    for (I i = 0; i < n; i++) o.peritab[o.permtab[i]] = i;
    // supernodes were recorded top-down: reverse them into elimination order
    o.rangtab.assign(cn + 1, 0);
    VI d(cn);
    for (I i = 0; i < cn; i++) {
        o.rangtab[i + 1] = rang[cn - i - 1] + 1;
        d[i] = depth[cn - i - 1];
    }
    // father = first later supernode that is shallower
    o.treetab.assign(cn, -1);
    std::vector<I> stack;
    for (I i = cn - 1; i >= 0; i--) {
        while (!stack.empty() && d[stack.back()] >= d[i]) stack.pop_back();
        o.treetab[i] = stack.empty() ? d[i] : stack.back();
        stack.push_back(i);
    }
    o.treetab[cn - 1] = -1;
}

// ---------------------------------------------------------------- step 2 --
void apply_level_order(Ordering &o, I width2d) {
    const I cn = o.cblknbr;
    if (cn <= 1) return;
    // sons of every node in increasing order; roots are the sons of -1
    VI nsons(cn + 1, 0), sonptr(cn + 2, 0), sons(cn);
    for (I i = 0; i < cn; i++) nsons[o.treetab[i] + 1]++;
    for (I i = 0; i <= cn; i++) sonptr[i + 1] = sonptr[i] + nsons[i];
    {
        VI pos(sonptr.begin(), sonptr.end() - 1);
        for (I i = 0; i < cn; i++) sons[pos[o.treetab[i] + 1]++] = i;
    }
    auto nsonsof = [&](I node) { return nsons[node + 1]; };
    auto sonof = [&](I node, I s) { return sons[sonptr[node + 1] + s]; };

    std::vector<int8_t> is2d(cn, 0);
    I tot2d = 0;
    for (I node = cn - 1; node >= 0; node--) {
        const I f = o.treetab[node];
        const I size = o.rangtab[node + 1] - o.rangtab[node];
        if (size >= width2d && (f == -1 || (is2d[f] && nsonsof(f) == 2))) {
            is2d[node] = 1;
            tot2d++;
        }
    }
    VI sorted(cn), newfath(cn, -1);
    I pos2d = 0, pos1d = tot2d;
    for (I s = 0; s < nsonsof(-1); s++) {
        I node = sonof(-1, s);
        if (is2d[node]) sorted[pos2d++] = node; else sorted[pos1d++] = node;
    }
    for (I i = 0; i < cn; i++) {
        const I node = sorted[i];
        const I ns = nsonsof(node);
        I s2 = 0;
        for (I s = 0; s < ns; s++) s2 += is2d[sonof(node, s)];
        const I s1 = ns - s2;
        I c2 = 0, c1 = 0;
        for (I s = 0; s < ns; s++) {
            const I son = sonof(node, s);
            if (is2d[son]) sorted[pos2d + s2 - c2++ - 1] = son;
            else sorted[pos1d + s1 - c1++ - 1] = son;
            newfath[son] = cn - i - 1;
        }
        pos2d += s2;
        pos1d += s1;
    }
    VI rang(cn + 1, 0), tree(cn), peri(o.n);
    for (I i = 0; i < cn; i++) {
        const I node = sorted[cn - i - 1];
        const I size = o.rangtab[node + 1] - o.rangtab[node];
        rang[i + 1] = rang[i] + size;
        tree[i] = newfath[node];
        std::copy(o.peritab.begin() + o.rangtab[node], o.peritab.begin() + o.rangtab[node] + size,
                  peri.begin() + rang[i]);
    }
    o.rangtab.swap(rang);
    o.treetab.swap(tree);
    o.peritab.swap(peri);
    for (I i = 0; i < o.n; i++) o.permtab[o.peritab[i]] = i;
}

// ---------------------------------------------------------------- step 3 --
// Block structure of L for the supernode partition: rows of cblk k are the
// neighbours of its columns beyond it plus what its elimination-tree
// children contribute beyond it; blocks are maximal runs of consecutive rows
// inside one facing cblk.
struct Graph {
    I n;
    VI ptr, adj;   // symmetrised, no diagonal
};

void symbolic_fax(const Graph &g, const Ordering &o, Symbol &s) {
    const I cn = o.cblknbr;
    s = Symbol();
    s.cblknbr = cn;
    s.nodenbr = o.n;
    s.fcol.resize(cn);
    s.lcol.resize(cn);
    s.bloknum.assign(cn + 1, 0);
    std::vector<VI> rows(cn);          // off-diagonal rows of each cblk, sorted
    std::vector<VI> chain(cn);         // contributing children
    VI mark(o.n, -1);
    VI col2cblk(o.n);
    for (I k = 0; k < cn; k++)
        for (I c = o.rangtab[k]; c < o.rangtab[k + 1]; c++) col2cblk[c] = k;
    for (I k = 0; k < cn; k++) {
        const I colmax = o.rangtab[k + 1];
        VI r;
        for (I col = o.rangtab[k]; col < colmax; col++) {
            const I v = o.peritab[col];
            for (I e = g.ptr[v]; e < g.ptr[v + 1]; e++) {
                const I ce = o.permtab[g.adj[e]];
                if (ce >= colmax && mark[ce] != k) {
                    mark[ce] = k;
                    r.push_back(ce);
                }
            }
        }
        for (I ch : chain[k])
            for (I ce : rows[ch])
                if (ce >= colmax && mark[ce] != k) {
                    mark[ce] = k;
                    r.push_back(ce);
                }
        std::sort(r.begin(), r.end());
        s.fcol[k] = o.rangtab[k];
        s.lcol[k] = colmax - 1;
        s.bloknum[k] = (I)s.frow.size();
        s.frow.push_back(o.rangtab[k]);
        s.lrow.push_back(colmax - 1);
        s.lcblk.push_back(k);
        s.fcblk.push_back(k);
        for (size_t i = 0; i < r.size();) {
            const I f = col2cblk[r[i]];
            size_t j = i + 1;
            while (j < r.size() && r[j] == r[j - 1] + 1 && r[j] < o.rangtab[f + 1]) j++;
            s.frow.push_back(r[i]);
            s.lrow.push_back(r[j - 1]);
            s.lcblk.push_back(k);
            s.fcblk.push_back(f);
            i = j;
        }
        if (!r.empty()) chain[col2cblk[r[0]]].push_back(k);
        rows[k].swap(r);
        chain[k].clear();
        chain[k].shrink_to_fit();
    }
    s.bloknbr = (I)s.frow.size();
    s.bloknum[cn] = s.bloknbr;
    s.build_rowtab();
}

// ---------------------------------------------------------------- step 4 --
I hamming(const std::vector<VI> &vec, I xi, I xj, I stop) {
    if (xi == -1) return (I)vec[xj].size();
    if (xj == -1) return (I)vec[xi].size();
    const VI &a = vec[xi], &b = vec[xj];
    const I sa = (I)a.size(), sb = (I)b.size();
    if (sa - sb >= stop || sb - sa >= stop) return stop;
    I sum = 0, i = 0, j = 0;
    while (i < sa && j < sb) {
        if (a[i] == b[j]) {
            i++;
            j++;
        } else if (a[i] < b[j]) {
            while (i < sa && a[i] < b[j]) {
                sum++;
                i++;
            }
        } else {
            while (j < sb && a[i] > b[j]) {
                sum++;
                j++;
            }
        }
        if (sum >= stop) return stop;
    }
    sum += (sa - i) + (sb - j);
    return sum >= stop ? stop : sum;
}

// Insert the rows of one supernode one after the other in the cyclic tour
// (with a ghost row) at the position that lengthens it least.
void reorder_tsp(I size, I *peri, const std::vector<VI> &lw, const std::vector<VI> &up, I stop) {
    if (size < 3) return;
    VI inv(size + 1), len(size + 1, 0);
    inv[0] = -1;
    inv[1] = 0;
    I d = hamming(lw, 0, -1, stop);
    len[0] = d;
    len[1] = d;
    for (I i = 1; i < size; i++) {
        I lwb = hamming(lw, i, inv[0], stop);
        I lwa = hamming(lw, i, inv[1], stop);
        I upa = hamming(up, i, inv[1], 1);
        I minl = lwb + lwa - len[0];
        I mpos = 1;
        I mincut = -1;
        for (I j = 1; j < i; j++) {
            const I upb = upa;
            upa = hamming(up, i, inv[j + 1], 1);
            if (upb < 1 || upa < 1) {
                if (lwa == -1) lwb = hamming(lw, i, inv[j], stop);
                else lwb = lwa;
                lwa = hamming(lw, i, inv[j + 1], stop);
                const I l = lwb + lwa - len[j];
                if (l == minl) {
                    if (lwb < mincut) {
                        mincut = lwb;
                        minl = l;
                        mpos = j + 1;
                    }
                    if (lwa < mincut) {
                        mincut = lwa;
                        minl = l;
                        mpos = j + 1;
                    }
                }
                if (l < minl) {
                    mincut = lwb;
                    minl = l;
                    mpos = j + 1;
                    if (lwa < mincut) mincut = lwa;
                }
                if (lwa == 0) {
                    mincut = 0;
                    minl = l;
                    mpos = j + 1;
                    j = i;
                }
            } else {
                lwa = -1;
            }
        }
        const I firstp = hamming(lw, i, inv[0], stop);
        const I lastp = hamming(lw, i, inv[i], stop);
        lwb = hamming(lw, i, inv[mpos - 1], stop);
        lwa = hamming(lw, i, inv[mpos], stop);
        const I l = firstp + lastp - len[i];
        if (l < minl) {
            minl = l;
            mpos = i + 1;
        }
        if (mpos > 0) len[mpos - 1] = lwb;
        if (mpos < i + 1) {
            I k = i, ll = lwa;
            for (I j = mpos; j < i + 2; j++) {
                std::swap(inv[j], k);
                std::swap(len[j], ll);
            }
        } else {
            inv[i + 1] = i;
            len[i + 1] = firstp;
        }
    }
    I elected = 0;
    for (I i = 0; i < size; i++)
        if (inv[i] == -1) elected = i;
    VI tmp(size);
    for (I i = 0; i < size; i++) tmp[i] = peri[inv[(i + 1 + elected) % (size + 1)]];
    std::copy(tmp.begin(), tmp.end(), peri);
}

void symbol_reordering(const Symbol &s, Ordering &o, I split_level, I stop) {
    const I cn = s.cblknbr;
    VI levels(cn, 0);
    I maxdepth = 0;
    for (I i = 0; i < cn; i++) {
        I l = 1, f = o.treetab[i];
        while (f != -1) {
            l++;
            f = o.treetab[f];
        }
        levels[i] = l;
        maxdepth = std::max(maxdepth, l);
    }
    VI dw(maxdepth);
    for (I k = 0; k < cn; k++) {
        const I size = s.lcol[k] - s.fcol[k] + 1;
        std::fill(dw.begin(), dw.end(), 0);
        for (I it = s.brownum[k]; it < s.brownum[k + 1]; it++) {
            const I b = s.browtab[it];
            dw[levels[s.lcblk[b]] - 1] += s.lrow[b] - s.frow[b] + 1;
        }
        I lsl = split_level;
        {
            I sign = 0;
            for (;;) {
                I upt = 0, lwt = 0, i = 0;
                for (; i < lsl; i++) upt += dw[i];
                for (; i < maxdepth; i++) lwt += dw[i];
                if (lwt < 5 * upt && lwt > 10 && upt > 10 && sign <= 0) {
                    lsl--;
                    sign--;
                    continue;
                }
                if (lwt > 3 * upt && lwt > 10 && upt > 10 && sign >= 0) {
                    lsl++;
                    sign++;
                    continue;
                }
                break;
            }
        }
        std::vector<VI> up(size), lw(size);
        for (I it = s.brownum[k]; it < s.brownum[k + 1]; it++) {
            const I b = s.browtab[it];
            auto &dst = (levels[s.lcblk[b]] <= lsl) ? up : lw;
            for (I r = s.frow[b]; r <= s.lrow[b]; r++) dst[r - s.fcol[k]].push_back(s.lcblk[b]);
        }
        reorder_tsp(size, o.peritab.data() + o.rangtab[k], lw, up, stop);
    }
    for (I i = 0; i < o.n; i++) o.permtab[o.peritab[i]] = i;
}

// ---------------------------------------------------------------- step 5 --
I iceil(I a, I b) { return (a + b - 1) / b; }

I nb_split(I width, I bmin, I bmax) {
    if (width <= bmax) return 1;
    I nseq = iceil(width, bmax);
    if (nseq > 1 && width / nseq < bmin) nseq--;
    return nseq;
}

// split point (relative to the first column) that cuts the fewest blocks in
// a window of +-10% around the even split
I smallest_split(const I *nbl, I step, I mn, I mx, I percent) {
    const I limit = iceil(step * percent, 100);
    if (step >= mx) return mx - 1;
    const I avg = step - 1;
    const I lmin = std::max(avg - limit - 1, mn);
    const I lmax = std::min(avg + limit + 1, mx);
    I best = avg, nb = nbl[avg];
    for (I i = avg + 1; i < lmax; i++)
        if (nbl[i] < nb) {
            best = i;
            nb = nbl[i];
        }
    for (I i = avg - 1; i > lmin; i--)
        if (nbl[i] < nb) {
            best = i;
            nb = nbl[i];
        }
    return best;
}

void split_symbol(Symbol &s, I bmin, I bmax) {
    const I cn = s.cblknbr;
    VI sptcblk(cn, -1), sptcbnb(cn, 1);
    VI exf, exl;   // extra cblks
    I addcblk = 0;
    VI nbl;        // blocks crossing the row pair (r, r+1), indexed r - fsplit
    I fsplit = -1;
    for (I k = 0; k < cn; k++) {
        I width = s.lcol[k] - s.fcol[k] + 1;
        if (nb_split(width, bmin, bmax) <= 1) continue;
        if (fsplit < 0) {
            fsplit = s.fcol[k];
            nbl.assign(s.nodenbr - fsplit + 1, 0);
            for (I b = 0; b < s.bloknbr; b++) {
                if (s.lrow[b] < fsplit) continue;
                for (I line = std::max(s.frow[b], fsplit); line < s.lrow[b]; line++) nbl[line - fsplit]++;
            }
        }
        I nb = 0;
        I fc = s.fcol[k];
        while (fc <= s.lcol[k]) {
            const I nseq = nb_split(width, bmin, bmax);
            if (nseq == 1) {
                exf.push_back(fc);
                exl.push_back(s.lcol[k]);
                nb++;
                fc = s.lcol[k] + 1;
                continue;
            }
            const I step = iceil(width, nseq);
            const I lwidth = width - bmin;
            const I lc = fc + smallest_split(nbl.data() + (fc - fsplit), step, bmin, lwidth, 10);
            exf.push_back(fc);
            exl.push_back(lc);
            nb++;
            width -= lc - fc + 1;
            fc = lc + 1;
        }
        addcblk += nb - 1;
        sptcblk[k] = (I)exf.size() - nb;
        sptcbnb[k] = nb;
        for (I b = s.bloknum[k] + 1; b < s.bloknum[k + 1]; b++)
            for (I line = s.frow[b]; line < s.lrow[b]; line++) nbl[line - fsplit] += nb - 1;
    }
    if (addcblk == 0) return;

    Symbol t;
    t.cblknbr = cn + addcblk;
    t.nodenbr = s.nodenbr;
    VI newnum(cn + 1, 0);
    for (I k = 0; k < cn; k++) newnum[k + 1] = newnum[k] + sptcbnb[k];
    VI extranew(exf.size(), -1);
    t.fcol.resize(t.cblknbr);
    t.lcol.resize(t.cblknbr);
    for (I k = 0; k < cn; k++) {
        if (sptcbnb[k] > 1) {
            for (I j = 0; j < sptcbnb[k]; j++) {
                extranew[sptcblk[k] + j] = newnum[k] + j;
                t.fcol[newnum[k] + j] = exf[sptcblk[k] + j];
                t.lcol[newnum[k] + j] = exl[sptcblk[k] + j];
            }
        } else {
            t.fcol[newnum[k]] = s.fcol[k];
            t.lcol[newnum[k]] = s.lcol[k];
        }
    }
    t.bloknum.assign(t.cblknbr + 1, 0);
    I cur = 0;
    for (I k = 0; k < cn; k++) {
        const I w = sptcbnb[k];
        for (I j = 0; j < w; j++, cur++) {
            t.bloknum[cur] = (I)t.frow.size();
            for (I q = 0; q < w - j; q++) {
                t.frow.push_back(t.fcol[cur + q]);
                t.lrow.push_back(t.lcol[cur + q]);
                t.lcblk.push_back(cur);
                t.fcblk.push_back(cur + q);
            }
            for (I b = s.bloknum[k] + 1; b < s.bloknum[k + 1]; b++) {
                I fr = s.frow[b];
                const I lr = s.lrow[b], f = s.fcblk[b];
                if (sptcbnb[f] > 1) {
                    for (I l = 0; l < sptcbnb[f]; l++) {
                        const I nf = sptcblk[f] + l;
                        if (fr > exl[nf]) continue;
                        if (lr < exf[nf]) break;
                        t.frow.push_back(fr);
                        t.lrow.push_back(std::min(lr, exl[nf]));
                        t.lcblk.push_back(cur);
                        t.fcblk.push_back(extranew[sptcblk[f]] + l);
                        fr = exl[nf] + 1;
                    }
                } else {
                    t.frow.push_back(fr);
                    t.lrow.push_back(lr);
                    t.lcblk.push_back(cur);
                    t.fcblk.push_back(newnum[f]);
                }
            }
        }
    }
    t.bloknbr = (I)t.frow.size();
    t.bloknum[t.cblknbr] = t.bloknbr;
    t.build_rowtab();
    s = std::move(t);
}

}  // namespace

// ------------------------------------------------------------------ C ABI --
struct pastix_gpu_analysis_s {
    Ordering order;     // final ordering
    Symbol symb;        // final (split) symbol = solver cblk/blok tables
    I ocblknbr = 0;     // supernodes of the ordering (before the split)
};

extern "C" int pastix_gpu_analyze_grid(pastix_gpu_analysis_t **out, int64_t nx, int64_t ny, int64_t nz,
                                       int64_t n, const int64_t *colptr, const int64_t *rowptr,
                                       const int64_t *iparm) {
    if (!out || nx <= 0 || ny <= 0 || nz <= 0 || nx * ny * nz != n || !colptr || !rowptr)
        return PASTIX_GPU_ERR_BADPARAMETER;
    *out = nullptr;
    I bmin = 160, bmax = 320, width2d = -1, rsplit = 0, rstop = INT64_MAX;
    if (iparm) {
        bmin = iparm[36];
        bmax = iparm[37];
        width2d = iparm[39];
        rsplit = iparm[28];
        rstop = iparm[29];
    }
    if (width2d < 0) width2d = bmin;
    if (bmin <= 0 || bmax < bmin) return PASTIX_GPU_ERR_BADPARAMETER;
    // symmetrised graph without the diagonal (graph/graph_prepare.c:115)
    Graph g;
    g.n = n;
    g.ptr.assign(n + 1, 0);
    for (I j = 0; j < n; j++)
        for (I k = colptr[j]; k < colptr[j + 1]; k++) {
            const I i = rowptr[k];
            if (i < 0 || i >= n) return PASTIX_GPU_ERR_BADPARAMETER;
            if (i != j) {
                g.ptr[i + 1]++;
                g.ptr[j + 1]++;
            }
        }
    for (I i = 0; i < n; i++) g.ptr[i + 1] += g.ptr[i];
    g.adj.assign(g.ptr[n], 0);
    {
        VI pos(g.ptr.begin(), g.ptr.end() - 1);
        for (I j = 0; j < n; j++)
            for (I k = colptr[j]; k < colptr[j + 1]; k++) {
                const I i = rowptr[k];
                if (i != j) {
                    g.adj[pos[i]++] = j;
                    g.adj[pos[j]++] = i;
                }
            }
        for (I i = 0; i < n; i++) {
            std::sort(g.adj.begin() + g.ptr[i], g.adj.begin() + g.ptr[i + 1]);
            // merge duplicates (both triangles given)
            auto b = g.adj.begin() + g.ptr[i], e = g.adj.begin() + g.ptr[i + 1];
            auto u = std::unique(b, e);
            std::fill(u, e, -1);
        }
        // compact
        VI np(n + 1, 0), na;
        na.reserve(g.adj.size());
        for (I i = 0; i < n; i++) {
            for (I e = g.ptr[i]; e < g.ptr[i + 1]; e++)
                if (g.adj[e] >= 0) na.push_back(g.adj[e]);
            np[i + 1] = (I)na.size();
        }
        g.ptr.swap(np);
        g.adj.swap(na);
    }
    auto *an = new pastix_gpu_analysis_s();
    order_grid(nx, ny, nz, an->order);
    apply_level_order(an->order, width2d);
    an->ocblknbr = an->order.cblknbr;
    Symbol s;
    symbolic_fax(g, an->order, s);
    symbol_reordering(s, an->order, rsplit, rstop);
    symbolic_fax(g, an->order, s);
    split_symbol(s, bmin, bmax);
    an->symb = std::move(s);
    *out = an;
    return PASTIX_GPU_SUCCESS;
}

// Structure handoff through files: the SolverMatrix written by the
// reference's solverSave (blend/solver_io.c:261: header "2", then cblknbr,
// bloknbr, nodenbr, baseval, one {fcolnum, lcolnum, first blok} line per
// cblk and one {frownum, lrownum, fcblknm} line per blok; what follows --
// coefficient offsets, tasks -- is not needed on the GPU) and the ordering
// written by pastixOrderSave (order/order_io.c:199 ordering_save: header
// "1", then cblknbr, vertnbr, rangtab, permtab, treetab).  The owner cblk of
// each blok follows from the cblks' first bloks, the blocks facing each cblk
// (browtab) from the bloks' facing cblks.
static bool read_ints(FILE *f, I count, VI &out) {
    out.resize(count);
    for (I k = 0; k < count; k++) {
        long v;
        if (fscanf(f, "%ld", &v) != 1) return false;
        out[k] = v;
    }
    return true;
}

extern "C" int pastix_gpu_analysis_load(pastix_gpu_analysis_t **out, const char *solver_file,
                                        const char *order_file) {
    if (!out || !solver_file || !order_file) return PASTIX_GPU_ERR_BADPARAMETER;
    *out = nullptr;
    std::unique_ptr<pastix_gpu_analysis_t> an(new pastix_gpu_analysis_t());
    // the ordering
    FILE *fo = fopen(order_file, "r");
    if (!fo) return PASTIX_GPU_ERR_BADPARAMETER;
    VI hdr;
    bool ok = read_ints(fo, 3, hdr) && hdr[0] == 1 && hdr[1] > 0 && hdr[2] > 0;
    Ordering &o = an->order;
    if (ok) {
        o.cblknbr = hdr[1];
        o.n = hdr[2];
        ok = read_ints(fo, o.cblknbr + 1, o.rangtab) && read_ints(fo, o.n, o.permtab) &&
             read_ints(fo, o.cblknbr, o.treetab);
    }
    fclose(fo);
    if (!ok) return PASTIX_GPU_ERR_BADPARAMETER;
    const I obase = o.rangtab[0];
    if (obase != 0 && obase != 1) return PASTIX_GPU_ERR_BADPARAMETER;
    for (auto &v : o.rangtab) v -= obase;
    for (auto &v : o.permtab) v -= obase;
    o.peritab.assign(o.n, -1);
    for (I i = 0; i < o.n; i++) {
        if (o.permtab[i] < 0 || o.permtab[i] >= o.n || o.peritab[o.permtab[i]] >= 0) return PASTIX_GPU_ERR_BADPARAMETER;
        o.peritab[o.permtab[i]] = i;
    }
    an->ocblknbr = o.cblknbr;
    // the solver matrix
    FILE *fs = fopen(solver_file, "r");
    if (!fs) return PASTIX_GPU_ERR_BADPARAMETER;
    Symbol &sy = an->symb;
    ok = read_ints(fs, 5, hdr) && hdr[0] == 2 && hdr[1] > 0 && hdr[2] >= hdr[1] && hdr[3] == o.n &&
         (hdr[4] == 0 || hdr[4] == 1);
    VI ctab, btab;
    if (ok) {
        sy.cblknbr = hdr[1];
        sy.bloknbr = hdr[2];
        sy.nodenbr = hdr[3];
        ok = read_ints(fs, 3 * sy.cblknbr, ctab) && read_ints(fs, 3 * sy.bloknbr, btab);
    }
    fclose(fs);
    if (!ok) return PASTIX_GPU_ERR_BADPARAMETER;
    const I base = hdr[4];
    sy.fcol.resize(sy.cblknbr);
    sy.lcol.resize(sy.cblknbr);
    sy.bloknum.resize(sy.cblknbr + 1);
    for (I c = 0; c < sy.cblknbr; c++) {
        sy.fcol[c] = ctab[3 * c] - base;
        sy.lcol[c] = ctab[3 * c + 1] - base;
        sy.bloknum[c] = ctab[3 * c + 2];
    }
    sy.bloknum[sy.cblknbr] = sy.bloknbr;
    sy.frow.resize(sy.bloknbr);
    sy.lrow.resize(sy.bloknbr);
    sy.fcblk.resize(sy.bloknbr);
    sy.lcblk.resize(sy.bloknbr);
    for (I b = 0; b < sy.bloknbr; b++) {
        sy.frow[b] = btab[3 * b] - base;
        sy.lrow[b] = btab[3 * b + 1] - base;
        sy.fcblk[b] = btab[3 * b + 2] - base;
    }
    for (I c = 0; c < sy.cblknbr; c++) {
        if (sy.bloknum[c] < 0 || sy.bloknum[c] >= sy.bloknum[c + 1] || sy.lcol[c] < sy.fcol[c])
            return PASTIX_GPU_ERR_BADPARAMETER;
        for (I b = sy.bloknum[c]; b < sy.bloknum[c + 1]; b++) {
            if (sy.fcblk[b] < 0 || sy.fcblk[b] >= sy.cblknbr) return PASTIX_GPU_ERR_BADPARAMETER;
            sy.lcblk[b] = c;
        }
    }
    if (sy.lcol[sy.cblknbr - 1] + 1 != o.n) return PASTIX_GPU_ERR_BADPARAMETER;
    sy.build_rowtab();
    *out = an.release();
    return PASTIX_GPU_SUCCESS;
}

extern "C" int pastix_gpu_analysis_sizes(const pastix_gpu_analysis_t *an, int64_t *sizes) {
    if (!an || !sizes) return PASTIX_GPU_ERR_BADPARAMETER;
    sizes[0] = an->order.n;
    sizes[1] = an->symb.cblknbr;
    sizes[2] = an->symb.bloknbr;
    sizes[3] = (int64_t)an->symb.browtab.size();
    sizes[4] = an->ocblknbr;
    return PASTIX_GPU_SUCCESS;
}

extern "C" int pastix_gpu_analysis_export(const pastix_gpu_analysis_t *an, int64_t *cblktab, int64_t *bloktab,
                                          int64_t *browtab, int64_t *permtab, int64_t *peritab,
                                          int64_t *rangtab, int64_t *treetab) {
    if (!an) return PASTIX_GPU_ERR_BADPARAMETER;
    const Symbol &s = an->symb;
    if (cblktab) {
        for (I c = 0; c < s.cblknbr; c++) {
            cblktab[4 * c + 0] = s.fcol[c];
            cblktab[4 * c + 1] = s.lcol[c];
            cblktab[4 * c + 2] = s.bloknum[c];
            cblktab[4 * c + 3] = s.brownum[c];
        }
        const I c = s.cblknbr;
        cblktab[4 * c + 0] = s.lcol[c - 1] + 1;
        cblktab[4 * c + 1] = s.lcol[c - 1] + 1;
        cblktab[4 * c + 2] = s.bloknbr;
        cblktab[4 * c + 3] = s.brownum[c];
    }
    if (bloktab)
        for (I b = 0; b < s.bloknbr; b++) {
            bloktab[4 * b + 0] = s.frow[b];
            bloktab[4 * b + 1] = s.lrow[b];
            bloktab[4 * b + 2] = s.lcblk[b];
            bloktab[4 * b + 3] = s.fcblk[b];
        }
    if (browtab) std::copy(s.browtab.begin(), s.browtab.end(), browtab);
    if (permtab) std::copy(an->order.permtab.begin(), an->order.permtab.end(), permtab);
    if (peritab) std::copy(an->order.peritab.begin(), an->order.peritab.end(), peritab);
    if (rangtab) std::copy(an->order.rangtab.begin(), an->order.rangtab.end(), rangtab);
    if (treetab) std::copy(an->order.treetab.begin(), an->order.treetab.end(), treetab);
    return PASTIX_GPU_SUCCESS;
}

extern "C" void pastix_gpu_analysis_free(pastix_gpu_analysis_t **an) {
    if (an && *an) {
        delete *an;
        *an = nullptr;
    }
}
