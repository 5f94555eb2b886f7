// compile.cpp — plan compilation: SQL-level expression nodes → typed IR
// (the planner's translation, planner/physical.go:376-818), accumulator slot
// layout (exec/aggregate.go:51-72, 255-279), group-key encoding, zone-map
// predicate (planner/physical.go:624-750), and generation of the query-
// specialised sm_100a scan kernels compiled at plan creation.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <limits>
#include <numeric>
#include <set>
#include <sstream>

#include "plan.h"

namespace vq {

// ---- dates: time.ParseInLocation("2006-01-02", s, time.UTC) --------------------
bool parse_date(const char* s, int64_t* days) {
    if (!s || std::strlen(s) != 10 || s[4] != '-' || s[7] != '-') return false;
    int digits[8] = {0, 1, 2, 3, 5, 6, 8, 9};
    for (int i : digits) if (s[i] < '0' || s[i] > '9') return false;
    int y = (s[0] - '0') * 1000 + (s[1] - '0') * 100 + (s[2] - '0') * 10 + (s[3] - '0');
    int m = (s[5] - '0') * 10 + (s[6] - '0');
    int d = (s[8] - '0') * 10 + (s[9] - '0');
    static const int mdays[12] = {31, 28, 31, 30, 31, 30, 31, 31, 30, 31, 30, 31};
    if (m < 1 || m > 12 || d < 1) return false;
    bool leap = (y % 4 == 0 && y % 100 != 0) || y % 400 == 0;
    if (d > mdays[m - 1] + ((m == 2 && leap) ? 1 : 0)) return false;
    // days since 1970-01-01 by counting whole years and months
    int64_t n = 0;
    auto isLeap = [](int yy) { return (yy % 4 == 0 && yy % 100 != 0) || yy % 400 == 0; };
    if (y >= 1970) for (int yy = 1970; yy < y; yy++) n += isLeap(yy) ? 366 : 365;
    else for (int yy = y; yy < 1970; yy++) n -= isLeap(yy) ? 366 : 365;
    for (int mm = 1; mm < m; mm++) n += mdays[mm - 1] + ((mm == 2 && leap) ? 1 : 0);
    *days = n + d - 1;
    return true;
}

namespace {

// likeMatch semantics of exec/expr.go:1277-1311 (% any run, _ one byte)
bool like_match(const char* p, size_t pn, const char* s, size_t sn) {
    while (pn > 0) {
        if (*p == '%') {
            p++; pn--;
            if (pn == 0) return true;
            for (size_t i = 0; i <= sn; i++)
                if (like_match(p, pn, s + i, sn - i)) return true;
            return false;
        }
        if (sn == 0) return false;
        if (*p != '_' && *p != *s) return false;
        p++; pn--; s++; sn--;
    }
    return sn == 0;
}

struct Translator {
    Plan& p;
    const vexq_expr* nodes;
    int nnodes;
    const int32_t* children;
    int nchildren;
    Table* t;        // column scope: the scan table
    Table* bt;       // joined scope: build table (columns [0, nbuild))
    int nbuild = 0;
    bool joined = false;
    std::vector<std::pair<int, int64_t>>* presence = nullptr;  // presence rows of the scanned table
    std::vector<std::string> lit_strs;  // per IR node (string literals)

    const vexq_expr& at(int i) const {
        if (i < 0 || i >= nnodes) fail(VEXQ_EINVAL, "expression node index out of range");
        return nodes[i];
    }
    int child(const vexq_expr& n, int k) const {
        int idx = n.child0 + k;
        if (k >= n.nchildren || idx < 0 || idx >= nchildren) fail(VEXQ_EINVAL, "expression child out of range");
        return children[idx];
    }
    int add(INode n) {
        p.ir.push_back(std::move(n));
        lit_strs.resize(p.ir.size());
        return (int)p.ir.size() - 1;
    }
    INode& N(int i) { return p.ir[i]; }

    const Column& colref(int c, bool build) const {
        const Table* tt = build ? bt : t;
        return tt->cols[c];
    }

    int lit_node(int type) {
        INode n;
        n.k = NK::Lit;
        n.type = type;
        return add(n);
    }

    // coerceOneSide (planner/physical.go:782-818): coerce literal b to a's type.
    int coerce(int a, int b) {
        if (N(b).k != NK::Lit) return b;
        int at_ = N(a).type, bt_ = N(b).type;
        if (at_ == VEXQ_TYPE_DATE) {
            if (bt_ == VEXQ_TYPE_STRING) {
                int64_t days;
                if (parse_date(lit_strs[b].c_str(), &days)) {
                    int n = lit_node(VEXQ_TYPE_DATE);
                    N(n).ld = (int32_t)days;
                    return n;
                }
            } else if (bt_ == VEXQ_TYPE_INT64) {
                int n = lit_node(VEXQ_TYPE_DATE);
                N(n).ld = (int32_t)N(b).li;
                return n;
            }
        } else if (at_ == VEXQ_TYPE_FLOAT64 && bt_ == VEXQ_TYPE_INT64) {
            int n = lit_node(VEXQ_TYPE_FLOAT64);
            N(n).lf = (double)N(b).li;
            return n;
        } else if (at_ == VEXQ_TYPE_INT64 && bt_ == VEXQ_TYPE_FLOAT64) {
            double f = N(b).lf;
            int n = lit_node(VEXQ_TYPE_INT64);
            N(n).li = (std::isnan(f) || f >= 9.2233720368547758e18 || f < -9.2233720368547758e18)
                          ? std::numeric_limits<int64_t>::min() : (int64_t)f;
            return n;
        }
        return b;
    }

    int bool_node(NK k, std::vector<int> ch) {
        INode n;
        n.k = k;
        n.type = VEXQ_TYPE_BOOL;
        n.ch = std::move(ch);
        return add(n);
    }

    int cmp_node(int op, int l, int r) {
        int lt = N(l).type, rt = N(r).type;
        if (lt != rt || lt == VEXQ_TYPE_STRING || lt == VEXQ_TYPE_BOOL)
            fail(VEXQ_EINVAL, "comparison operands are not comparable (expr: cmp not supported)");
        INode n;
        n.k = NK::Cmp;
        n.type = VEXQ_TYPE_BOOL;
        n.op = op;
        n.ch = {l, r};
        return add(n);
    }

    int cast_float(int e) {
        if (N(e).type != VEXQ_TYPE_INT64) return e;
        INode n;
        n.k = NK::Cast;
        n.type = VEXQ_TYPE_FLOAT64;
        n.ch = {e};
        return add(n);
    }

    int string_col_of(int e) {
        if (N(e).k != NK::Col || N(e).type != VEXQ_TYPE_STRING)
            fail(VEXQ_ENOTSUP, "string predicate over a non-column operand");
        return e;
    }

    // buildExecExpr (planner/physical.go:376-547) + buildBinExpr (:549-620)
    int tr(int idx) {
        const vexq_expr& n = at(idx);
        switch (n.kind) {
            case VEXQ_E_COLUMN: {
                INode c;
                c.k = NK::Col;
                int ci = n.column;
                if (joined) {
                    if (ci < 0 || ci >= nbuild + (int)t->cols.size()) fail(VEXQ_EINVAL, "column index out of range");
                    if (ci < nbuild) c.build = true;
                    else ci -= nbuild;
                } else if (ci < 0 || ci >= (int)t->cols.size()) {
                    fail(VEXQ_EINVAL, "column index out of range");
                }
                c.col = ci;
                c.tab = c.build ? bt : t;
                const Column& col = colref(ci, c.build);
                c.type = col.type;
                c.nullable = col.nullable;
                return add(c);
            }
            case VEXQ_E_LITERAL: {
                INode c;
                c.k = NK::Lit;
                c.is_literal_raw = true;
                c.lit_kind = n.lit_kind;
                std::string s;
                switch (n.lit_kind) {
                    case VEXQ_LIT_INT: c.type = VEXQ_TYPE_INT64; c.li = n.lit_int; break;
                    case VEXQ_LIT_FLOAT: c.type = VEXQ_TYPE_FLOAT64; c.lf = n.lit_float; break;
                    case VEXQ_LIT_STRING: c.type = VEXQ_TYPE_STRING; s = n.lit_str ? n.lit_str : ""; break;
                    case VEXQ_LIT_BOOL: c.type = VEXQ_TYPE_BOOL; c.lb = n.lit_int != 0; break;
                    default: fail(VEXQ_EINVAL, "bad literal kind");
                }
                int id = add(c);
                lit_strs[id] = s;
                return id;
            }
            case VEXQ_E_AND:
            case VEXQ_E_OR: {
                std::vector<int> ch;
                for (int k = 0; k < n.nchildren; k++) {
                    int c = tr(child(n, k));
                    if (N(c).type != VEXQ_TYPE_BOOL) fail(VEXQ_EINVAL, "AND/OR operand is not boolean");
                    ch.push_back(c);
                }
                if (ch.empty()) {  // empty AND → all true; empty OR → all false (valid)
                    int l = lit_node(VEXQ_TYPE_BOOL);
                    N(l).lb = n.kind == VEXQ_E_AND;
                    return l;
                }
                return bool_node(n.kind == VEXQ_E_AND ? NK::And : NK::Or, ch);
            }
            case VEXQ_E_NOT: {
                int c = tr(child(n, 0));
                if (N(c).type != VEXQ_TYPE_BOOL) fail(VEXQ_EINVAL, "NOT requires a boolean operand");
                return bool_node(NK::Not, {c});
            }
            case VEXQ_E_NEG: {  // physical.go:414-436: child * -1
                int c = tr(child(n, 0));
                int t_ = N(c).type;
                if (t_ != VEXQ_TYPE_FLOAT64 && t_ != VEXQ_TYPE_INT64) fail(VEXQ_EINVAL, "unary minus not supported for type");
                int l = lit_node(t_);
                N(l).lf = -1.0;
                N(l).li = -1;
                INode a;
                a.k = NK::Arith;
                a.op = VEXQ_OP_MUL;
                a.type = t_;
                a.ch = {c, l};
                return add(a);
            }
            case VEXQ_E_IS_NULL:
            case VEXQ_E_IS_NOT_NULL:
                return bool_node(n.kind == VEXQ_E_IS_NULL ? NK::IsNull : NK::IsNotNull, {tr(child(n, 0))});
            case VEXQ_E_BETWEEN: {  // BetweenExpr → AND(GE, LE) (exec/expr.go:1328-1339)
                int c = tr(child(n, 0));
                int lo = coerce(c, tr(child(n, 1)));
                int hi = coerce(c, tr(child(n, 2)));
                int a = bool_node(NK::And, {cmp_node(VEXQ_OP_GE, c, lo), cmp_node(VEXQ_OP_LE, c, hi)});
                return n.op == 1 ? bool_node(NK::Not, {a}) : a;
            }
            case VEXQ_E_IN: {  // InExpr (exec/expr.go:1204-1243)
                int c = tr(child(n, 0));
                int kind = 0;
                std::vector<int64_t> si;
                std::vector<double> sf;
                std::vector<std::string> ss;
                for (int k = 1; k < n.nchildren; k++) {
                    const vexq_expr& l = at(child(n, k));
                    if (l.kind != VEXQ_E_LITERAL) continue;
                    int lk = l.lit_kind == VEXQ_LIT_INT ? 1 : l.lit_kind == VEXQ_LIT_FLOAT ? 2 : l.lit_kind == VEXQ_LIT_STRING ? 3 : 0;
                    if (!lk) continue;
                    if (kind && kind != lk) fail(VEXQ_EINVAL, "IN list mixes literal types");
                    kind = lk;
                    if (lk == 1) si.push_back(l.lit_int);
                    if (lk == 2) sf.push_back(l.lit_float);
                    if (lk == 3) ss.push_back(l.lit_str ? l.lit_str : "");
                }
                int ct = N(c).type;
                if (kind && ((ct == VEXQ_TYPE_INT64 && kind != 1) || (ct == VEXQ_TYPE_FLOAT64 && kind != 2) ||
                             (ct == VEXQ_TYPE_STRING && kind != 3)))
                    fail(VEXQ_EINVAL, "IN literal type does not match the operand");
                INode x;
                x.type = VEXQ_TYPE_BOOL;
                x.ch = {c};
                if (!kind || ct == VEXQ_TYPE_DATE || ct == VEXQ_TYPE_BOOL) {
                    x.k = NK::InFalse;  // no literal matches these vector kinds
                } else if (ct == VEXQ_TYPE_INT64) {
                    x.k = NK::InInt;
                    x.seti = si;
                } else if (ct == VEXQ_TYPE_FLOAT64) {
                    x.k = NK::InFloat;
                    x.setf = sf;
                } else {
                    string_col_of(c);
                    const Column& col = colref(N(c).col, N(c).build);
                    x.k = NK::InCodes;
                    x.col = N(c).col;
                    x.build = N(c).build;
                    x.codes.assign(col.dict.keys.size(), 0);
                    for (auto& s : ss) {
                        int64_t code = col.dict.find(s);
                        if (code >= 0) x.codes[code] = 1;
                    }
                }
                int id = add(x);
                return n.op == 1 ? bool_node(NK::Not, {id}) : id;
            }
            case VEXQ_E_LIKE: {  // LikeExpr: evaluated once per dictionary entry
                int c = tr(child(n, 0));
                const vexq_expr& pt = at(child(n, 1));
                if (pt.kind != VEXQ_E_LITERAL || pt.lit_kind != VEXQ_LIT_STRING)
                    fail(VEXQ_EINVAL, "LIKE pattern must be a string literal");
                if (N(c).type != VEXQ_TYPE_STRING) fail(VEXQ_EINVAL, "LIKE requires STRING column");
                string_col_of(c);
                std::string pat = pt.lit_str ? pt.lit_str : "";
                const Column& col = colref(N(c).col, N(c).build);
                INode x;
                x.k = NK::InCodes;
                x.type = VEXQ_TYPE_BOOL;
                x.ch = {c};
                x.col = N(c).col;
                x.build = N(c).build;
                x.codes.assign(col.dict.keys.size(), 0);
                for (size_t i = 0; i < col.dict.keys.size(); i++)
                    x.codes[i] = like_match(pat.data(), pat.size(), col.dict.keys[i].data(), col.dict.keys[i].size());
                int id = add(x);
                return n.op == 1 ? bool_node(NK::Not, {id}) : id;
            }
            case VEXQ_E_CASE: {  // CaseExpr (exec/expr.go:1405-1432), physical.go:508-546
                bool has_else = n.op == 1;
                int nw = (n.nchildren - (has_else ? 1 : 0)) / 2;
                INode x;
                x.k = NK::Case;
                x.has_else = has_else;
                for (int w = 0; w < nw; w++) {
                    int cond = tr(child(n, 2 * w));
                    int res = tr(child(n, 2 * w + 1));
                    x.ch.push_back(cond);
                    x.ch.push_back(res);
                }
                if (has_else) x.ch.push_back(tr(child(n, n.nchildren - 1)));
                int t_ = nw > 0 ? N(x.ch[1]).type : VEXQ_TYPE_FLOAT64;
                for (int w = 0; w < nw; w++) {
                    if (N(x.ch[2 * w]).type != VEXQ_TYPE_BOOL) fail(VEXQ_EINVAL, "CASE condition is not boolean");
                    if (N(x.ch[2 * w + 1]).type != t_) fail(VEXQ_EINVAL, "CASE branches must have a common type");
                }
                if (has_else && N(x.ch.back()).type != t_) fail(VEXQ_EINVAL, "CASE ELSE type mismatch");
                if (t_ != VEXQ_TYPE_INT64 && t_ != VEXQ_TYPE_FLOAT64)
                    fail(VEXQ_ENOTSUP, "CASE with a non-numeric result type is not supported on the GPU path");
                x.type = t_;
                return add(x);
            }
            case VEXQ_E_BINARY: {
                int l = tr(child(n, 0));
                int r = tr(child(n, 1));
                l = coerce(r, l);  // coercePair: both directions (physical.go:773-778)
                r = coerce(l, r);
                if ((n.op == VEXQ_OP_EQ || n.op == VEXQ_OP_NE) && N(l).type == VEXQ_TYPE_STRING &&
                    N(r).type == VEXQ_TYPE_STRING) {
                    int cidx = -1, lidx = -1;
                    if (N(l).k == NK::Col && N(r).k == NK::Lit) { cidx = l; lidx = r; }
                    else if (N(r).k == NK::Col && N(l).k == NK::Lit) { cidx = r; lidx = l; }
                    if (cidx < 0) fail(VEXQ_EINVAL, "expr: cmp not supported for string operands");
                    // StringEqExpr (exec/expr.go:1342-1388)
                    INode x;
                    x.k = NK::StrEq;
                    x.type = VEXQ_TYPE_BOOL;
                    x.col = N(cidx).col;
                    x.build = N(cidx).build;
                    x.negate = n.op == VEXQ_OP_NE;
                    x.ch = {cidx};
                    const Column& col = colref(x.col, x.build);
                    x.streq_code = col.dict.find(lit_strs[lidx]);
                    if (x.streq_code >= 0 && !x.build && col.per_rg_dicts) {
                        bool all = true;
                        for (auto& pr : col.rg_present) if (!pr[x.streq_code]) { all = false; break; }
                        if (!all) {
                            std::vector<std::pair<int, int64_t>>& pl = presence ? *presence : p.presence;
                            x.present_idx = (int)pl.size();
                            pl.push_back({x.col, x.streq_code});
                        }
                    }
                    return add(x);
                }
                if (n.op < VEXQ_OP_EQ || n.op > VEXQ_OP_DIV) fail(VEXQ_EINVAL, "unknown binary op");
                if (n.op <= VEXQ_OP_GE) return cmp_node(n.op, l, r);
                int rt = N(l).type;
                if (N(l).type == VEXQ_TYPE_FLOAT64 || N(r).type == VEXQ_TYPE_FLOAT64) rt = VEXQ_TYPE_FLOAT64;
                if (rt == VEXQ_TYPE_FLOAT64) { l = cast_float(l); r = cast_float(r); }
                if (N(l).type != N(r).type || (N(l).type != VEXQ_TYPE_INT64 && N(l).type != VEXQ_TYPE_FLOAT64))
                    fail(VEXQ_EINVAL, "arithmetic operand types not supported (missing plan-time coercion?)");
                INode a;
                a.k = NK::Arith;
                a.op = n.op;
                a.type = rt;
                a.ch = {l, r};
                return add(a);
            }
        }
        fail(VEXQ_EINVAL, "unsupported expression kind");
    }
};

// Static NULL-ability and |value| bounds (interval arithmetic over the
// table-wide min/max of each column) of every IR node.
void analyze(Plan& p) {
    for (size_t i = 0; i < p.ir.size(); i++) {
        INode& n = p.ir[i];
        auto C = [&](int k) -> INode& { return p.ir[n.ch[k]]; };
        switch (n.k) {
            case NK::Col: {
                const Table* tt = n.tab ? n.tab : (n.build ? p.bt : p.t);
                const Column& c = tt->cols[n.col];
                n.nullable = c.nullable;
                if (c.has_range) {
                    n.bounded = true;
                    if (c.type == VEXQ_TYPE_FLOAT64) { n.lo = c.fmin; n.hi = c.fmax; }
                    else { n.lo = (double)c.imin; n.hi = (double)c.imax; }
                    if (!std::isfinite(n.lo) || !std::isfinite(n.hi)) n.bounded = false;
                } else if (c.type == VEXQ_TYPE_BOOL) {
                    n.bounded = true; n.lo = 0; n.hi = 1;
                }
                n.finite = c.type != VEXQ_TYPE_FLOAT64 || (c.finite && n.bounded);
                break;
            }
            case NK::Lit:
                n.nullable = false;
                n.bounded = true;
                n.lo = n.hi = n.type == VEXQ_TYPE_FLOAT64 ? n.lf : n.type == VEXQ_TYPE_DATE ? n.ld : (double)n.li;
                if (!std::isfinite(n.lo)) n.bounded = false;
                n.finite = n.type != VEXQ_TYPE_FLOAT64 || n.bounded;
                break;
            case NK::Cast:
                n.nullable = C(0).nullable;
                n.bounded = C(0).bounded; n.lo = C(0).lo; n.hi = C(0).hi;
                n.finite = C(0).finite || C(0).type != VEXQ_TYPE_FLOAT64;
                break;
            case NK::Arith: {
                n.nullable = C(0).nullable || C(1).nullable;
                n.bounded = C(0).bounded && C(1).bounded;
                if (!n.bounded) break;
                double a = C(0).lo, b = C(0).hi, c = C(1).lo, d = C(1).hi;
                switch (n.op) {
                    case VEXQ_OP_ADD: n.lo = a + c; n.hi = b + d; break;
                    case VEXQ_OP_SUB: n.lo = a - d; n.hi = b - c; break;
                    case VEXQ_OP_MUL: {
                        double v[4] = {a * c, a * d, b * c, b * d};
                        n.lo = *std::min_element(v, v + 4);
                        n.hi = *std::max_element(v, v + 4);
                        break;
                    }
                    case VEXQ_OP_DIV: {
                        if (n.type == VEXQ_TYPE_INT64) { n.lo = -std::max(std::fabs(a), std::fabs(b)); n.hi = -n.lo; break; }
                        if (c <= 0 && d >= 0) { n.bounded = false; break; }
                        double v[4] = {a / c, a / d, b / c, b / d};
                        n.lo = *std::min_element(v, v + 4);
                        n.hi = *std::max_element(v, v + 4);
                        break;
                    }
                }
                if (n.bounded && (!std::isfinite(n.lo) || !std::isfinite(n.hi))) n.bounded = false;
                // widen by a relative ulp margin for rounding
                if (n.bounded) { double m = std::max(std::fabs(n.lo), std::fabs(n.hi)) * 1e-12; n.lo -= m; n.hi += m; }
                // finite operands inside finite bounds give a finite result
                n.finite = n.type != VEXQ_TYPE_FLOAT64 || (n.bounded && C(0).finite && C(1).finite);
                break;
            }
            case NK::Case: {
                int nw = (int)(n.ch.size() - (n.has_else ? 1 : 0)) / 2;
                n.nullable = !n.has_else;
                n.bounded = true;
                n.lo = INFINITY; n.hi = -INFINITY;
                for (int w = 0; w <= nw; w++) {
                    int ri = w < nw ? n.ch[2 * w + 1] : (n.has_else ? n.ch.back() : -1);
                    if (ri < 0) continue;
                    const INode& r = p.ir[ri];
                    n.nullable = n.nullable || r.nullable;
                    if (!r.bounded) { n.bounded = false; continue; }
                    n.lo = std::min(n.lo, r.lo);
                    n.hi = std::max(n.hi, r.hi);
                }
                if (!n.has_else) { n.lo = std::min(n.lo, 0.0); n.hi = std::max(n.hi, 0.0); }
                n.finite = true;
                for (int w = 0; w <= nw; w++) {
                    int ri = w < nw ? n.ch[2 * w + 1] : (n.has_else ? n.ch.back() : -1);
                    if (ri >= 0 && !p.ir[ri].finite) n.finite = false;
                }
                n.finite = n.finite || n.type != VEXQ_TYPE_FLOAT64;
                break;
            }
            case NK::IsNull:
            case NK::IsNotNull:
                n.nullable = false;
                n.finite = true;
                break;
            case NK::StrEq:
                n.nullable = C(0).nullable || n.present_idx >= 0 || n.streq_code < 0;
                n.finite = true;
                break;
            case NK::StrRank:
                n.nullable = C(0).nullable;
                n.bounded = true;
                n.lo = 0;
                n.hi = n.rank.empty() ? 0.0 : (double)(n.rank.size() - 1);
                n.finite = true;
                break;
            default: {
                bool any = false;
                for (int c : n.ch) any = any || p.ir[c].nullable;
                n.nullable = any;
                n.finite = n.type != VEXQ_TYPE_FLOAT64;
                break;
            }
        }
    }
}

std::string ctype(int t) {
    switch (t) {
        case VEXQ_TYPE_INT64: return "long long";
        case VEXQ_TYPE_FLOAT64: return "double";
        case VEXQ_TYPE_DATE: return "int";
        case VEXQ_TYPE_STRING: return "unsigned";
        case VEXQ_TYPE_BOOL: return "bool";
    }
    return "long long";
}

std::string dlit(double v) {  // exact double literal (bit cast keeps NaN payloads)
    int64_t b;
    std::memcpy(&b, &v, 8);
    std::ostringstream o;
    o << "__longlong_as_double(" << b << "LL)";
    return o.str();
}

std::string ilit(int64_t v) {
    if (v == std::numeric_limits<int64_t>::min()) return "(-9223372036854775807LL - 1LL)";
    return std::to_string(v) + "LL";
}

const char* cmp_op(int op) {
    switch (op) {
        case VEXQ_OP_EQ: return "==";
        case VEXQ_OP_NE: return "!=";
        case VEXQ_OP_LT: return "<";
        case VEXQ_OP_LE: return "<=";
        case VEXQ_OP_GT: return ">";
        case VEXQ_OP_GE: return ">=";
    }
    return "==";
}

// Emits straight-line code for IR nodes, memoised per scope.
struct Gen {
    Plan& p;
    std::ostringstream& os;
    std::vector<char> done;
    std::string ind = "            ";
    // scanned-table columns: from the chunk registers (cv/cm), or gathered at
    // row `row` (partition join, where rows arrive one by one)
    bool gather = false;
    std::string row = "r";
    // partition join: probe columns carried in the payload, read at entry `pay_row`
    const std::vector<int>* pay_slot = nullptr;
    std::string pay_row = "e";
    // index of the current row in a chunk column (cv<c>[kidx]): "k" for the
    // register arrays, "(k << 5)" for strided reads of a staged chunk
    std::string kidx = "k";
    Gen(Plan& pp, std::ostringstream& o) : p(pp), os(o), done(pp.ir.size(), 0) {}

    void emit(int i) {
        if (done[i]) return;
        INode& n = p.ir[i];
        for (int c : n.ch) emit(c);
        done[i] = 1;
        std::string x = "x" + std::to_string(i), ok = "ok" + std::to_string(i);
        auto X = [&](int k) { return "x" + std::to_string(n.ch[k]); };
        auto OK = [&](int k) { return "ok" + std::to_string(n.ch[k]); };
        switch (n.k) {
            case NK::Col: {
                std::string c = std::to_string(n.col);
                if (n.build) {
                    std::string ct = n.type == VEXQ_TYPE_BOOL ? "unsigned char" : ctype(n.type);
                    os << ind << "const bool " << ok << " = " << (n.nullable ? "vq_bit(P.bvalid[" + c + "], brow)" : "true") << ";\n";
                    std::string ld = "((const " + ct + "*)P.bcol[" + c + "])[brow]";
                    if (n.type == VEXQ_TYPE_BOOL)  // a NULL bool reads false
                        os << ind << "const bool " << x << " = " << ok << " && " << ld << " != 0;\n";
                    else
                        os << ind << "const " << ctype(n.type) << " " << x << " = " << ld << ";\n";
                } else if (gather && pay_slot && n.col < (int)pay_slot->size() && (*pay_slot)[n.col] >= 0) {
                    const std::string j = std::to_string((*pay_slot)[n.col]);
                    os << ind << "const bool " << ok << " = " << (n.nullable ? "P.qpayv[" + j + "][" + pay_row + "] != 0" : "true") << ";\n";
                    const std::string w = "P.qpay[" + j + "][" + pay_row + "]";
                    switch (n.type) {
                        case VEXQ_TYPE_FLOAT64: os << ind << "const double " << x << " = __longlong_as_double((long long)" << w << ");\n"; break;
                        case VEXQ_TYPE_INT64: os << ind << "const long long " << x << " = (long long)" << w << ";\n"; break;
                        case VEXQ_TYPE_DATE: os << ind << "const int " << x << " = (int)(long long)" << w << ";\n"; break;
                        case VEXQ_TYPE_STRING: os << ind << "const unsigned " << x << " = (unsigned)" << w << ";\n"; break;
                        default: os << ind << "const bool " << x << " = " << ok << " && " << w << " != 0ull;\n"; break;
                    }
                } else if (gather) {
                    std::string ct = n.type == VEXQ_TYPE_BOOL ? "unsigned char" : ctype(n.type);
                    os << ind << "const bool " << ok << " = " << (n.nullable ? "vq_bit(P.valid[" + c + "], " + row + ")" : "true") << ";\n";
                    std::string ld = "((const " + ct + "*)P.col[" + c + "])[" + row + "]";
                    if (n.type == VEXQ_TYPE_BOOL)
                        os << ind << "const bool " << x << " = " << ok << " && " << ld << " != 0;\n";
                    else
                        os << ind << "const " << ctype(n.type) << " " << x << " = " << ld << ";\n";
                } else {
                    os << ind << "const bool " << ok << " = " << (n.nullable ? "((cm" + c + " >> k) & 1u) != 0u" : "true") << ";\n";
                    if (n.type == VEXQ_TYPE_BOOL)
                        os << ind << "const bool " << x << " = " << ok << " && cv" << c << "[" << kidx << "] != 0u;\n";
                    else
                        os << ind << "const " << ctype(n.type) << " " << x << " = cv" << c << "[" << kidx << "];\n";
                }
                break;
            }
            case NK::Lit: {
                os << ind << "const bool " << ok << " = true;\n";
                if (n.lit_slot >= 0) {  // value passed at launch
                    std::string L = "P.lit[" + std::to_string(n.lit_slot) + "]";
                    if (n.type == VEXQ_TYPE_INT64) os << ind << "const long long " << x << " = " << L << ";\n";
                    else if (n.type == VEXQ_TYPE_FLOAT64) os << ind << "const double " << x << " = __longlong_as_double(" << L << ");\n";
                    else os << ind << "const int " << x << " = (int)" << L << ";\n";
                    break;
                }
                switch (n.type) {
                    case VEXQ_TYPE_INT64: os << ind << "const long long " << x << " = " << ilit(n.li) << ";\n"; break;
                    case VEXQ_TYPE_FLOAT64: os << ind << "const double " << x << " = " << dlit(n.lf) << ";\n"; break;
                    case VEXQ_TYPE_DATE: os << ind << "const int " << x << " = " << n.ld << ";\n"; break;
                    case VEXQ_TYPE_BOOL: os << ind << "const bool " << x << " = " << (n.lb ? "true" : "false") << ";\n"; break;
                    default: os << ind << "const unsigned " << x << " = 0u;\n"; break;
                }
                break;
            }
            case NK::Cmp:
                os << ind << "const bool " << ok << " = " << OK(0) << " && " << OK(1) << ";\n";
                os << ind << "const bool " << x << " = " << ok << " && (" << X(0) << " " << cmp_op(n.op) << " " << X(1) << ");\n";
                break;
            case NK::Arith: {
                os << ind << "const bool " << ok << " = " << OK(0) << " && " << OK(1) << ";\n";
                if (n.type == VEXQ_TYPE_FLOAT64) {
                    std::string e;
                    switch (n.op) {
                        case VEXQ_OP_ADD: e = X(0) + " + " + X(1); break;
                        case VEXQ_OP_SUB: e = X(0) + " - " + X(1); break;
                        case VEXQ_OP_MUL: e = X(0) + " * " + X(1); break;
                        case VEXQ_OP_DIV:  // applyArithFloat64: x/0 → math.NaN()
                            e = "(" + X(1) + " == 0.0 ? __longlong_as_double(0x7FF8000000000001LL) : " + X(0) + " / " + X(1) + ")";
                            break;
                    }
                    os << ind << "const double " << x << " = " << ok << " ? (" << e << ") : 0.0;\n";
                } else {
                    std::string a = "(unsigned long long)" + X(0), b = "(unsigned long long)" + X(1), e;
                    switch (n.op) {
                        case VEXQ_OP_ADD: e = "(long long)(" + a + " + " + b + ")"; break;
                        case VEXQ_OP_SUB: e = "(long long)(" + a + " - " + b + ")"; break;
                        case VEXQ_OP_MUL: e = "(long long)(" + a + " * " + b + ")"; break;
                        case VEXQ_OP_DIV:
                            e = "(" + X(1) + " == 0LL ? 0LL : (" + X(1) + " == -1LL ? (long long)(0ull - " + a + ") : " + X(0) +
                                " / " + X(1) + "))";
                            break;
                    }
                    os << ind << "const long long " << x << " = " << ok << " ? " << e << " : 0LL;\n";
                }
                break;
            }
            case NK::Cast:
                os << ind << "const bool " << ok << " = " << OK(0) << ";\n";
                os << ind << "const double " << x << " = (double)" << X(0) << ";\n";
                break;
            case NK::And:
            case NK::Or: {
                const char* o = n.k == NK::And ? " & " : " | ";
                os << ind << "const bool " << x << " = ";
                for (size_t k = 0; k < n.ch.size(); k++) os << (k ? o : "") << X((int)k);
                os << ";\n" << ind << "const bool " << ok << " = ";
                for (size_t k = 0; k < n.ch.size(); k++) os << (k ? o : "") << OK((int)k);
                os << ";\n";
                break;
            }
            case NK::Not:  // NotExpr: flip only valid bits (exec/expr.go:1134-1137)
                os << ind << "const bool " << ok << " = " << OK(0) << ";\n";
                os << ind << "const bool " << x << " = " << X(0) << " != " << OK(0) << ";\n";
                break;
            case NK::IsNull:
            case NK::IsNotNull:
                os << ind << "const bool " << ok << " = true;\n";
                os << ind << "const bool " << x << " = " << (n.k == NK::IsNull ? "!" : "") << OK(0) << ";\n";
                break;
            case NK::InInt:
            case NK::InFloat: {
                os << ind << "const bool " << ok << " = " << OK(0) << ";\n";
                os << ind << "const bool " << x << " = " << OK(0) << " && (false";
                if (n.k == NK::InInt) for (auto v : n.seti) os << " || " << X(0) << " == " << ilit(v);
                else for (auto v : n.setf) os << " || " << X(0) << " == " << dlit(v);
                os << ");\n";
                break;
            }
            case NK::InFalse:
                os << ind << "const bool " << ok << " = " << OK(0) << ";\n";
                os << ind << "const bool " << x << " = false;\n";
                break;
            case NK::InCodes: {
                os << ind << "const bool " << ok << " = " << OK(0) << ";\n";
                if (n.codes.size() <= 64) {
                    uint64_t m = 0;
                    for (size_t c = 0; c < n.codes.size(); c++) if (n.codes[c]) m |= 1ull << c;
                    os << ind << "const bool " << x << " = " << OK(0) << " && " << X(0) << " < 64u && ((" << m << "ull >> "
                       << X(0) << ") & 1ull);\n";
                } else {
                    os << ind << "const bool " << x << " = " << OK(0) << " && ((__ldg(P.sets[" << n.set_idx << "] + ("
                       << X(0) << " >> 5)) >> (" << X(0) << " & 31u)) & 1u);\n";
                }
                break;
            }
            case NK::StrEq: {
                std::string neg = n.negate ? "true" : "false";
                if (n.streq_code < 0) {  // literal in no dictionary: no rows (= ) / all rows (<>)
                    os << ind << "const bool " << ok << " = " << neg << ";\n";
                    os << ind << "const bool " << x << " = " << neg << ";\n";
                    break;
                }
                std::string m = "(" + OK(0) + " && ((" + X(0) + " == " + std::to_string(n.streq_code) + "u) != " + neg + "))";
                if (n.present_idx < 0) {
                    os << ind << "const bool " << ok << " = " << OK(0) << ";\n";
                    os << ind << "const bool " << x << " = " << m << ";\n";
                } else {
                    os << ind << "const bool pr" << i << " = __ldg(P.present + " << n.present_idx
                       << " * P.n_rg + (int)(r / P.rg_rows)) != 0;\n";
                    os << ind << "const bool " << ok << " = pr" << i << " ? " << OK(0) << " : " << neg << ";\n";
                    os << ind << "const bool " << x << " = pr" << i << " ? " << m << " : " << neg << ";\n";
                }
                break;
            }
            case NK::StrRank:  // a NULL row reads rank 0; its slot update is skipped by ok
                os << ind << "const bool " << ok << " = " << OK(0) << ";\n";
                os << ind << "const long long " << x << " = " << ok << " ? (long long)__ldg(P.sets[" << n.set_idx << "] + "
                   << X(0) << ") : 0LL;\n";
                break;
            case NK::Case: {
                std::string t = ctype(n.type);
                int nw = (int)(n.ch.size() - (n.has_else ? 1 : 0)) / 2;
                os << ind << t << " " << x << " = " << (n.has_else ? X((int)n.ch.size() - 1) : std::string(n.type == VEXQ_TYPE_FLOAT64 ? "0.0" : "0LL")) << ";\n";
                os << ind << "bool " << ok << " = " << (n.has_else ? OK((int)n.ch.size() - 1) : std::string("false")) << ";\n";
                for (int w = nw - 1; w >= 0; w--)
                    os << ind << "if (" << OK(2 * w) << " && " << X(2 * w) << ") { " << x << " = " << X(2 * w + 1) << "; " << ok
                       << " = " << OK(2 * w + 1) << "; }\n";
                break;
            }
        }
    }
};

// Structural signature of an IR subtree (deduplicates accumulator slots).
std::string sig(const Plan& p, int i) {
    const INode& n = p.ir[i];
    std::ostringstream o;
    o << (int)n.k << ":" << n.type << ":" << n.op << ":" << n.col << ":" << n.build << ":" << n.li << ":";
    int64_t fb;
    std::memcpy(&fb, &n.lf, 8);
    o << fb << ":" << n.ld << ":" << n.lb << ":" << n.streq_code << ":" << n.negate << ":" << n.has_else << "(";
    for (int c : n.ch) o << sig(p, c) << ",";
    for (auto v : n.seti) o << v << ";";
    for (auto v : n.setf) o << v << ";";
    for (auto v : n.codes) o << (int)v;
    o << ")";
    return o.str();
}

int add_slot(Plan& p, std::map<std::string, int>& seen, SlotKind k, int input) {
    std::string key = std::to_string((int)k) + "|" + (input >= 0 ? sig(p, input) : std::string("*"));
    auto it = seen.find(key);
    if (it != seen.end()) return it->second;
    p.slots.push_back(Slot{k, input});
    seen[key] = (int)p.slots.size() - 1;
    return (int)p.slots.size() - 1;
}

// AccumTypeFor + output typing (exec/aggregate.go:51-72, 161-175, 780-876).
void plan_aggs(Plan& p, const std::vector<std::pair<int, int>>& aggs_ir, const vexq_agg_desc* aggs) {
    std::map<std::string, int> seen;
    add_slot(p, seen, S_CNT, -1);  // slot 0: group row count (COUNT(*))
    for (size_t j = 0; j < aggs_ir.size(); j++) {
        int kind = aggs_ir[j].first, in = aggs_ir[j].second;
        AggOut o;
        o.kind = kind;
        o.name = aggs[j].out_name ? aggs[j].out_name : "";
        if (kind < VEXQ_AGG_COUNT || kind > VEXQ_AGG_COUNT_DISTINCT) fail(VEXQ_EINVAL, "unknown aggregate kind");
        if (in < 0) {
            if (kind != VEXQ_AGG_COUNT) fail(VEXQ_EINVAL, "aggregate column not found in schema");
            o.value_slot = 0;
            o.nn_slot = 0;
            o.out_type = VEXQ_TYPE_INT64;
            p.outs.push_back(o);
            continue;
        }
        const INode& x = p.ir[in];
        if (kind == VEXQ_AGG_COUNT_DISTINCT) {
            // COUNT(DISTINCT x) (exec/aggregate.go:474-493, 810-823): a count of
            // the rows whose (group, x) pair is new to the plan's distinct set
            // number d; output like COUNT (never NULL). One set per distinct
            // input expression.
            const std::string key = "D|" + sig(p, in);
            auto it = seen.find(key);
            if (it == seen.end()) {
                if (p.ndist >= VQ_MAXDIST) fail(VEXQ_ENOTSUP, "more than 4 COUNT(DISTINCT) aggregates in one plan");
                Slot sl{S_NN, in};
                sl.dset = p.ndist++;
                p.slots.push_back(sl);
                it = seen.emplace(key, (int)p.slots.size() - 1).first;
            }
            o.kind = VEXQ_AGG_COUNT;
            o.value_slot = o.nn_slot = it->second;
            o.out_type = VEXQ_TYPE_INT64;
            p.outs.push_back(o);
            continue;
        }
        int nn = x.nullable ? add_slot(p, seen, S_NN, in) : 0;
        o.nn_slot = nn;
        switch (kind) {
            case VEXQ_AGG_COUNT:
                o.value_slot = nn;
                o.out_type = VEXQ_TYPE_INT64;
                break;
            case VEXQ_AGG_SUM:
                if (x.type == VEXQ_TYPE_STRING) fail(VEXQ_ENOTSUP, "SUM over a STRING column is not supported on the GPU path");
                if (x.type == VEXQ_TYPE_FLOAT64) { o.value_slot = add_slot(p, seen, S_FSUM, in); o.out_type = VEXQ_TYPE_FLOAT64; }
                else { o.value_slot = add_slot(p, seen, S_ISUM, in); o.out_type = VEXQ_TYPE_INT64; }
                break;
            case VEXQ_AGG_AVG:
                if (x.type == VEXQ_TYPE_STRING) fail(VEXQ_ENOTSUP, "AVG over a STRING column is not supported on the GPU path");
                o.value_slot = add_slot(p, seen, S_FSUM, in);
                o.out_type = VEXQ_TYPE_FLOAT64;
                break;
            case VEXQ_AGG_MIN:
            case VEXQ_AGG_MAX:
                if (x.type == VEXQ_TYPE_STRING) {
                    // MIN/MAX over strings (HashAggregate.strAccs, exec/aggregate.go:98-110;
                    // merged in mergePartialAgg, exec/parallel.go:283-297): Go compares
                    // strings byte by byte, so the dictionary is ranked in that order,
                    // the slot takes MIN/MAX of the rank, and the rank maps back to the code
                    if (x.k != NK::Col) fail(VEXQ_ENOTSUP, "MIN/MAX over a STRING expression that is not a column");
                    const Table* tt = x.tab ? x.tab : (x.build ? p.bt : p.t);
                    const GlobalDict& dict = tt->cols[x.col].dict;
                    std::vector<uint32_t> order(dict.keys.size());
                    std::iota(order.begin(), order.end(), 0u);
                    std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return dict.keys[a] < dict.keys[b]; });
                    INode r;
                    r.k = NK::StrRank;
                    r.type = VEXQ_TYPE_INT64;
                    r.col = x.col;
                    r.build = x.build;
                    r.tab = x.tab;
                    r.ch = {in};
                    r.rank.assign(order.size(), 0);
                    for (size_t k = 0; k < order.size(); k++) r.rank[order[k]] = (uint32_t)k;
                    p.ir.push_back(std::move(r));
                    const int rn = (int)p.ir.size() - 1;
                    o.value_slot = add_slot(p, seen, kind == VEXQ_AGG_MIN ? S_IMIN : S_IMAX, rn);
                    o.out_type = VEXQ_TYPE_STRING;
                    o.rank_code = order;
                    o.rank_dict = &dict;
                    break;
                }
                if (x.type == VEXQ_TYPE_FLOAT64)
                    o.value_slot = add_slot(p, seen, kind == VEXQ_AGG_MIN ? S_FMIN : S_FMAX, in);
                else
                    o.value_slot = add_slot(p, seen, kind == VEXQ_AGG_MIN ? S_IMIN : S_IMAX, in);
                o.out_type = x.type;
                break;
        }
        p.outs.push_back(o);
    }
}

// Group-key encoding: dense codes when every key column has a small domain.
void plan_keys(Plan& p) {
    int64_t dom = 1;
    bool dense = true;
    for (auto& k : p.keys) {
        const Table* tt = k.build ? p.bt : p.t;
        const Column& c = tt->cols[k.col];
        k.type = c.type;
        k.nullable = c.nullable;
        int64_t d = 0;
        int64_t nul = c.nullable ? 1 : 0;  // NULL takes the last code of a nullable column
        if (c.type == VEXQ_TYPE_STRING) d = std::max<int64_t>((int64_t)c.dict.keys.size(), 1) + nul;
        else if (c.type == VEXQ_TYPE_BOOL) d = 2 + nul;
        else if ((c.type == VEXQ_TYPE_DATE || c.type == VEXQ_TYPE_INT64) && c.has_range && c.imax - c.imin < (1 << 22)) {
            k.vmin = c.imin;
            d = c.imax - c.imin + 1 + nul;
        } else if (!c.has_range && (c.type == VEXQ_TYPE_DATE || c.type == VEXQ_TYPE_INT64)) {
            d = 1;  // all NULL
            k.nullable = true;
        }
        if (d <= 0) { dense = false; k.domain = 0; continue; }
        k.domain = d;
        if (dom <= (int64_t(1) << 40)) dom *= d;
    }
    p.domain = dense ? dom : 0;
    // packed-key layout for the hash path
    int shift = 0;
    for (auto& k : p.keys) {
        if (k.domain > 0) {
            int b = 0;
            while ((int64_t(1) << b) < k.domain) b++;
            k.bits = std::max(b, 1);
        } else if (k.type == VEXQ_TYPE_DATE) {
            k.bits = 33;
        } else {
            if (k.nullable) fail(VEXQ_ENOTSUP, "GROUP BY over a nullable 64-bit column is not supported on the GPU path");
            k.bits = 64;
        }
        k.shift = shift;
        shift += k.bits;
    }
    if (shift > 64 && !dense) fail(VEXQ_ENOTSUP, "GROUP BY key wider than 64 bits is not supported on the GPU path");
}

void choose_path(Plan& p) {
    int regs_per_group = 1;  // first-occurrence key
    for (auto& s : p.slots) regs_per_group += 1;
    int max_groups = 16, max_acc = 64;
    if (const char* e = std::getenv("VEXQ_TUNE")) {
        const char* a = std::strstr(e, "regs_groups=");
        if (a) max_groups = std::atoi(a + 12);
        const char* b = std::strstr(e, "regs_acc=");
        if (b) max_acc = std::atoi(b + 9);
    }
    if (p.domain > 0 && p.domain <= max_groups && p.domain * regs_per_group <= max_acc) p.path = AggPath::Regs;
    else if (p.domain > 0 && p.domain <= (int64_t(1) << 22)) p.path = AggPath::Dense;
    else p.path = AggPath::Hash;
    // bank layout
    p.slot_pos.assign(p.slots.size(), -1);
    p.nf = p.ni = 0;
    for (size_t s = 0; s < p.slots.size(); s++) {
        bool in_float = p.path == AggPath::Regs ? p.slots[s].is_float() : p.slots[s].kind == S_FSUM;
        p.slot_pos[s] = in_float ? p.nf++ : p.ni++;
    }
    p.fx_lsb.assign(std::max(p.nf, 1), 0);
    if (p.path != AggPath::Regs) {
        if (p.nf > 16) fail(VEXQ_ENOTSUP, "more than 16 float sums in one aggregate");
        for (size_t s = 0; s < p.slots.size(); s++) {
            if (p.slots[s].kind != S_FSUM) continue;
            const INode& x = p.ir[p.slots[s].input];
            double m = x.bounded ? std::max(std::fabs(x.lo), std::fabs(x.hi)) : 0;
            if (!x.bounded) fail(VEXQ_ENOTSUP, "float sum over an unbounded expression (division by a range containing 0)");
            int e = 0;
            if (m > 0) std::frexp(m, &e);  // |x| <= m < 2^e
            // values of magnitude ≥ 2^(e-45) keep every mantissa bit; the top 31
            // bits of the 128-bit window hold sums of 2^31 rows
            p.fx_lsb[p.slot_pos[s]] = e - 97;
        }
    }
}

// ---- code generation --------------------------------------------------------------------------

struct ColUse {
    std::set<int> scan;  // scanned-table columns loaded per 4-row vector
};

void collect_cols(const Plan& p, int i, std::set<int>& scan) {
    if (i < 0) return;
    const INode& n = p.ir[i];
    if (n.k == NK::Col && !n.build) scan.insert(n.col);
    for (int c : n.ch) collect_cols(p, c, scan);
}

// 128-bit loads of four consecutive rows of every referenced column into
// registers named <pfx><col>[4] (values) and <mpfx><col> (validity nibble).
void emit_loads(std::ostringstream& os, const Plan& p, const Table* t, const std::set<int>& cols,
                const std::string& pfx = "cv", const std::string& mpfx = "cm", const std::string& r0 = "r0",
                const std::string& ind = "        ", bool declare = true) {
    for (int c : cols) {
        const Column& col = t->cols[c];
        std::string C = std::to_string(c), V = pfx + C;
        const char* ty = "unsigned";
        const char* fn = "vq_ld4_u32";
        switch (col.type) {
            case VEXQ_TYPE_INT64: ty = "long long"; fn = "vq_ld4_i64"; break;
            case VEXQ_TYPE_FLOAT64: ty = "double"; fn = "vq_ld4_f64"; break;
            case VEXQ_TYPE_DATE: ty = "int"; fn = "vq_ld4_i32"; break;
            case VEXQ_TYPE_BOOL: ty = "unsigned"; fn = "vq_ld4_u8"; break;
        }
        os << ind;
        if (declare) os << ty << " " << V << "[4]; ";
        os << fn << "(P.col[" << C << "], " << r0 << ", " << V << ");\n";
        if (col.nullable) {
            os << ind;
            if (declare) os << "unsigned ";
            os << mpfx << C << " = vq_bits4(P.valid[" << C << "], " << r0 << ");\n";
        }
    }
    (void)p;
}

void emit_declare_regs(std::ostringstream& os, const Table* t, const std::set<int>& cols, const std::string& pfx,
                       const std::string& mpfx, const std::string& ind) {
    for (int c : cols) {
        const Column& col = t->cols[c];
        const char* ty = col.type == VEXQ_TYPE_INT64 ? "long long" : col.type == VEXQ_TYPE_FLOAT64 ? "double"
                       : col.type == VEXQ_TYPE_DATE ? "int" : "unsigned";
        os << ind << ty << " " << pfx << c << "[4];";
        if (col.nullable) os << " unsigned " << mpfx << c << " = 0u;";
        os << "\n";
    }
}

void emit_copy_regs(std::ostringstream& os, const Table* t, const std::set<int>& cols, const std::string& ind) {
    for (int c : cols) {
        os << ind << "cv" << c << "[0] = nx" << c << "[0]; cv" << c << "[1] = nx" << c << "[1]; cv" << c << "[2] = nx" << c
           << "[2]; cv" << c << "[3] = nx" << c << "[3];";
        if (t->cols[c].nullable) os << " cm" << c << " = nm" << c << ";";
        os << "\n";
    }
}

// Group-key expression: dense gid or packed key, plus "any key NULL".
void emit_key(std::ostringstream& os, const Plan& p, const std::vector<int>& key_nodes, const std::string& ind) {
    bool dense = p.path != AggPath::Hash;
    os << ind << "unsigned long long key = 0ull;\n" << ind << "bool anynull = false;\n";
    long long stride = 1;
    for (size_t i = 0; i < p.keys.size(); i++) {
        const KeyCol& k = p.keys[i];
        std::string x = "x" + std::to_string(key_nodes[i]), ok = "ok" + std::to_string(key_nodes[i]);
        std::string code;
        os << ind << "anynull = anynull || !" << ok << ";\n";
        if (k.domain > 0) {
            std::string nullc = k.nullable ? std::to_string(k.domain - 1) + "ull" : std::string("0ull");
            if (k.type == VEXQ_TYPE_STRING) code = "(" + ok + " ? (unsigned long long)" + x + " : " + nullc + ")";
            else if (k.type == VEXQ_TYPE_BOOL) code = "(" + ok + " ? (" + x + " ? 1ull : 0ull) : " + nullc + ")";
            else code = "(" + ok + " ? (unsigned long long)((long long)" + x + " - " + ilit(k.vmin) + ") : " + nullc + ")";
        } else if (k.type == VEXQ_TYPE_DATE) {
            code = "(" + ok + " ? (unsigned long long)(unsigned)" + x + " : 0x100000000ull)";
        } else if (k.type == VEXQ_TYPE_FLOAT64) {
            code = "(unsigned long long)__double_as_longlong(" + x + ")";
        } else {
            code = "(unsigned long long)" + x;
        }
        if (dense) {
            os << ind << "key += " << code << " * " << stride << "ull;\n";
            stride *= k.domain;
        } else {
            os << ind << "key |= " << code << (k.shift ? " << " + std::to_string(k.shift) : std::string()) << ";\n";
        }
    }
}

// Order key of a group's first row: reproduces HashAggregate's insertion order
// (exec/aggregate.go:409-457; agg_intkey.go:249-255: NULL-keyed rows take the
// string-key path and are appended before the int-key groups).
std::string order_expr(const Plan& p, const std::string& pos) {
    if (!p.intkey_order) return pos;
    return "((anynull ? 0ll : (1ll << 56)) | " + pos + ")";
}

// live: the expression that says the row is in the scan and passes the
// predicate, where the loop runs rows that do not (atomic paths).
void emit_slot_values(std::ostringstream& os, const Plan& p, const std::string& ind, const std::string& live = "true") {
    for (size_t s = 1; s < p.slots.size(); s++) {
        const Slot& sl = p.slots[s];
        const INode& x = p.ir[sl.input];
        std::string X = "x" + std::to_string(sl.input), OK = "ok" + std::to_string(sl.input);
        std::string S = std::to_string(s);
        if (sl.dset >= 0) {
            // COUNT(DISTINCT): strings by global code (one code a string),
            // other types by extractInt64's image (raw float bits, dates
            // sign-extended, bools 0/1)
            std::string img;
            switch (x.type) {
                case VEXQ_TYPE_FLOAT64: img = "(unsigned long long)__double_as_longlong(" + X + ")"; break;
                case VEXQ_TYPE_BOOL: img = "(" + X + " ? 1ull : 0ull)"; break;
                case VEXQ_TYPE_DATE: img = "(unsigned long long)(long long)" + X; break;
                default: img = "(unsigned long long)" + X; break;
            }
            const std::string d = std::to_string(sl.dset);
            os << ind << "const bool sok" << S << " = " << OK << " && (" << live << ") && vq_dset_insert(P.dkeys[" << d
               << "], P.dstate[" << d << "], P.dmask, key, " << img << ", P.error);\n";
            continue;
        }
        os << ind << "const bool sok" << S << " = " << OK << ";\n";
        if (sl.is_float() || sl.kind == S_FSUM) {
            os << ind << "const double sv" << S << " = (double)" << (x.type == VEXQ_TYPE_BOOL ? "(" + X + " ? 1 : 0)" : X) << ";\n";
        } else if (sl.kind != S_NN) {
            os << ind << "const long long sv" << S << " = (long long)" << (x.type == VEXQ_TYPE_BOOL ? "(" + X + " ? 1 : 0)" : X) << ";\n";
        }
    }
}

std::string acc_name(const Plan& p, int g, int s) {
    return (p.slots[s].is_float() ? "af" : "ai") + std::to_string(g) + "_" + std::to_string(p.slot_pos[s]);
}

static bool slot_rdx(const Plan& p, size_t s) { return s < p.rdx.size() && p.rdx[s]; }
static bool slot_rfma(const Plan& p, size_t s) { return s < p.rfma.size() && p.rfma[s]; }
static int slot_alias(const Plan& p, size_t s) { return s < p.ralias.size() ? p.ralias[s] : -1; }

// Register variable holding slot s of group g during the scan: an exact-double
// accumulator ("ad") for integer-valued sums, the aliased slot's variable for
// a slot sharing another's sum, else the slot's own typed accumulator.
std::string acc_var(const Plan& p, int g, int s) {
    int t = slot_alias(p, s) >= 0 ? slot_alias(p, s) : s;
    if (slot_rdx(p, t)) return "ad" + std::to_string(g) + "_" + std::to_string(t);
    return acc_name(p, g, t);
}

// Integer input under a value-preserving int→float cast (the same values).
static int strip_int_cast(const Plan& p, int i) {
    while (i >= 0 && p.ir[i].k == NK::Cast && p.ir[i].type == VEXQ_TYPE_FLOAT64 && !p.ir[i].ch.empty() &&
           p.ir[p.ir[i].ch[0]].type != VEXQ_TYPE_FLOAT64)
        i = p.ir[i].ch[0];
    return i;
}

static bool same_column(const Plan& p, int a, int b) {
    if (a == b) return true;
    const INode &x = p.ir[a], &y = p.ir[b];
    return x.k == NK::Col && y.k == NK::Col && x.col == y.col && x.build == y.build && x.tab == y.tab;
}

// Chooses the register-path accumulator forms of an aggregate scan plan
// (joins keep the plain forms: a probe row may match many build rows, so
// no per-accumulator row bound exists). Integer-valued sums become exact
// doubles when every partial sum stays within 2^53 (|value| bound × table
// rows), which makes the update one FMA and lets AVG over an integer column
// share SUM's accumulator; float sums of never-NaN/inf values use
// fma(v, hit, acc), which equals the selected add bit for bit (v·1 and v·0
// are exact, and the accumulator, starting at +0, is never -0).
static void choose_regs_forms(Plan& p) {
    const size_t n = p.slots.size();
    p.rdx.assign(n, 0);
    p.rfma.assign(n, 0);
    p.ralias.assign(n, -1);
    if (p.path != AggPath::Regs || p.is_join || !p.t) return;
    const double rows = (double)std::max<int64_t>(p.t->nrows, 1);
    const double lim = 9007199254740992.0;  // 2^53
    std::vector<int> val(n, -1);
    for (size_t s = 0; s < n; s++) {
        const Slot& sl = p.slots[s];
        if (sl.kind == S_CNT || sl.kind == S_NN) {
            p.rdx[s] = rows <= lim;
            continue;
        }
        if (sl.kind != S_ISUM && sl.kind != S_FSUM) continue;
        const int v = strip_int_cast(p, sl.input);
        const INode& x = p.ir[v];
        if (x.type == VEXQ_TYPE_FLOAT64) {
            if (sl.kind == S_FSUM && p.ir[sl.input].finite) p.rfma[s] = 1;
            continue;
        }
        if (!x.bounded) continue;
        const double m = std::max(std::fabs(x.lo), std::fabs(x.hi));
        if (m * rows <= lim) {
            p.rdx[s] = 1;
            val[s] = v;
        }
    }
    for (size_t s = 0; s < n; s++) {
        if (!p.rdx[s] || val[s] < 0) continue;
        for (size_t t = 0; t < s; t++)
            if (p.rdx[t] && val[t] >= 0 && p.ralias[t] < 0 && same_column(p, val[s], val[t])) {
                p.ralias[s] = (int)t;
                break;
            }
    }
}

// Register path: the per-block partials are merged inside the scan kernel
// (each block adds its partials into global accumulators, the last block to
// arrive writes the merged row) when every float accumulator is a SUM of
// finite, bounded values: those partials add exactly as fixed-point integers
// (the window of the dense path's exact sums), so the merged sums do not
// depend on the order in which blocks finish, and integer sums, MIN, MAX and
// first-row keys are order-free as atomics. Float MIN/MAX keep the merge
// kernel, whose fold in block order keeps the first of two equal extremes
// (+0 against -0), and so do plans whose blocks would add more than 128
// atomics. VEXQ_TUNE "rfuse=0" keeps the merge kernel for measurement,
// "rfuse=2" folds any eligible plan into the scan, "rcopies=K" sets the
// accumulator copies.
static void choose_regs_fused(Plan& p) {
    p.rfused = false;
    if (p.path != AggPath::Regs || p.is_join || !p.t || p.nf > 16) return;
    if (p.t->nrows > (int64_t(1) << 31)) return;  // the window holds sums of 2^31 rows
    int force = 1;
    if (const char* e = std::getenv("VEXQ_TUNE")) {
        const char* at = std::strstr(e, "rfuse=");
        if (at) force = std::atoi(at + 6);
    }
    if (force == 0) return;
    // atomics a block adds: up to three fixed-point digits a float sum, one
    // a counter. 6M-row scans: one group of 2 entries (5 atomics) 37.4 us in
    // the scan against 39.5 us with the merge kernel. Six groups of 8 (108,
    // the Q1 shape): every block arrives at once and the atomics on the same
    // few L2 lines serialise, so the blocks add into 8 copies of the
    // accumulators (block b into copy b % 8): 59.2 us against 63.2 us with
    // the merge kernel and 63.6 us with one copy (4, 16 copies: 59.8, 59.6;
    // the 5-atomic Q6 shape is fastest with one copy, 34.8 against 35.0 with
    // 8). Larger banks keep the merge kernel (unmeasured).
    const int64_t atomics = p.domain * (3 * (int64_t)p.nf + p.ni + 1);
    if (atomics > 128 && force != 2) return;
    std::vector<int> lsb(std::max(p.nf, 1), 0);
    for (size_t s = 0; s < p.slots.size(); s++) {
        const Slot& sl = p.slots[s];
        if (sl.kind == S_FMIN || sl.kind == S_FMAX) return;
        if (sl.kind != S_FSUM) continue;
        if (!p.rfma[s] && !p.rdx[s]) return;  // a sum that may meet NaN or inf
        const INode& x = p.ir[sl.input];
        if (!x.bounded || !std::isfinite(x.lo) || !std::isfinite(x.hi)) return;
        const double m = std::max(std::fabs(x.lo), std::fabs(x.hi));
        int e = 0;
        if (m > 0) std::frexp(m, &e);  // |x| <= m < 2^e
        lsb[p.slot_pos[s]] = e - 97;
    }
    p.fx_lsb = lsb;
    p.rfused = true;
    if (p.rcopies == 0) p.rcopies = atomics > 16 ? 8 : 1;
}

// The predicated update of an aggregate scan writes first-row keys only on a
// lane's first row of each group, so they live in a per-thread array (local
// memory, written at most once per group) instead of registers.
static bool regs_fo_local(const Plan& p) { return p.regs_pred && !p.is_join; }

// Register path: accumulators live in registers, one set per dense group.
void emit_regs_decl(std::ostringstream& os, const Plan& p) {
    if (regs_fo_local(p)) {
        os << "    unsigned vq_seen = 0u;\n";
        os << "    long long vq_fo[" << p.domain << "];\n";
        os << "#pragma unroll\n    for (int g = 0; g < " << p.domain << "; g++) vq_fo[g] = 0x7FFFFFFFFFFFFFFFLL;\n";
    }
    for (int64_t g = 0; g < p.domain; g++) {
        if (!regs_fo_local(p)) os << "    long long fo" << g << " = 0x7FFFFFFFFFFFFFFFLL;\n";
        for (size_t s = 0; s < p.slots.size(); s++) {
            if (slot_alias(p, s) >= 0) continue;
            if (slot_rdx(p, s)) {
                os << "    double " << acc_var(p, (int)g, (int)s) << " = 0.0;\n";
                continue;
            }
            const Slot& sl = p.slots[s];
            std::string init;
            switch (sl.kind) {
                case S_IMIN: init = "0x7FFFFFFFFFFFFFFFLL"; break;
                case S_IMAX: init = "(-0x7FFFFFFFFFFFFFFFLL - 1LL)"; break;
                case S_FMIN: init = "1.7976931348623157e308"; break;   // math.MaxFloat64 (aggregate.go:262)
                case S_FMAX: init = "-1.7976931348623157e308"; break;
                case S_FSUM: init = "0.0"; break;
                default: init = "0LL"; break;
            }
            os << "    " << (sl.is_float() ? "double " : "long long ") << acc_name(p, (int)g, (int)s) << " = " << init << ";\n";
        }
    }
}

void emit_regs_update(std::ostringstream& os, const Plan& p, const std::string& ind, const std::string& order) {
    os << ind << "switch ((int)key) {\n";
    for (int64_t g = 0; g < p.domain; g++) {
        os << ind << "case " << g << ": {\n";
        std::string in = ind + "    ";
        os << in << "fo" << g << " = min(fo" << g << ", " << order << ");\n";
        for (size_t s = 0; s < p.slots.size(); s++) {
            if (slot_alias(p, s) >= 0) continue;
            std::string a = acc_var(p, (int)g, (int)s), S = std::to_string(s);
            if (slot_rdx(p, s)) {
                switch (p.slots[s].kind) {
                    case S_CNT: os << in << a << " += 1.0;\n"; break;
                    case S_NN: os << in << "if (sok" << S << ") " << a << " += 1.0;\n"; break;
                    default: os << in << "if (sok" << S << ") " << a << " += (double)sv" << S << ";\n"; break;
                }
                continue;
            }
            switch (p.slots[s].kind) {
                case S_CNT: os << in << a << " += 1LL;\n"; break;
                case S_NN: os << in << "if (sok" << S << ") " << a << " += 1LL;\n"; break;
                case S_ISUM: os << in << "if (sok" << S << ") " << a << " = (long long)((unsigned long long)" << a
                                << " + (unsigned long long)sv" << S << ");\n"; break;
                case S_IMIN: os << in << "if (sok" << S << " && sv" << S << " < " << a << ") " << a << " = sv" << S << ";\n"; break;
                case S_IMAX: os << in << "if (sok" << S << " && sv" << S << " > " << a << ") " << a << " = sv" << S << ";\n"; break;
                case S_FSUM: os << in << "if (sok" << S << ") " << a << " += sv" << S << ";\n"; break;
                case S_FMIN: os << in << "if (sok" << S << " && sv" << S << " < " << a << ") " << a << " = sv" << S << ";\n"; break;
                case S_FMAX: os << in << "if (sok" << S << " && sv" << S << " > " << a << ") " << a << " = sv" << S << ";\n"; break;
            }
        }
        os << in << "break;\n" << ind << "}\n";
    }
    os << ind << "default: break;\n" << ind << "}\n";
}

// Branch-free register update: every group's accumulators are updated with a
// select on (gid == g), so the four rows a lane holds form independent
// dependency chains the scheduler can interleave (a switch serialises them).
// A lane meets its rows in increasing row order (chunks and tiles ascend per
// warp) and a group's order key rises with the row, so a group's first-row
// key is recorded once, on the lane's first row of that group, in a branch
// taken at most once per group and lane. Exact-double and finite float sums
// are one FMA against the group's 0/1 hit.
void emit_regs_update_pred(std::ostringstream& os, const Plan& p, const std::string& ind, const std::string& order) {
    os << ind << "const unsigned vq_k32 = (unsigned)key;\n";
    os << ind << "{ const unsigned vq_kb = vq_k32 < 32u ? (1u << vq_k32) : 0u;\n";
    os << ind << "  if (key < " << p.domain << "ull && !(vq_seen & vq_kb)) {\n";
    os << ind << "    vq_seen |= vq_kb;\n";
    os << ind << "    vq_fo[vq_k32] = " << order << ";\n";
    os << ind << "  } }\n";
    for (size_t s = 0; s < p.slots.size(); s++) {
        if (slot_alias(p, s) >= 0) continue;
        std::string S = std::to_string(s);
        const SlotKind k = p.slots[s].kind;
        if (slot_rdx(p, s)) {
            if (k == S_NN) os << ind << "const double vd" << S << " = sok" << S << " ? 1.0 : 0.0;\n";
            else if (k != S_CNT) os << ind << "const double vd" << S << " = sok" << S << " ? (double)sv" << S << " : 0.0;\n";
        } else if (slot_rfma(p, s)) {
            os << ind << "const double vd" << S << " = sok" << S << " ? sv" << S << " : 0.0;\n";
        }
    }
    for (int64_t g = 0; g < p.domain; g++) {
        std::string G = std::to_string(g);
        os << ind << "{ const bool h = vq_k32 == " << g << "u;\n";
        std::string in = ind + "  ";
        os << in << "const double hd = h ? 1.0 : 0.0;\n";
        for (size_t s = 0; s < p.slots.size(); s++) {
            if (slot_alias(p, s) >= 0) continue;
            std::string a = acc_var(p, (int)g, (int)s), S = std::to_string(s);
            if (slot_rdx(p, s) && p.slots[s].kind == S_CNT) {
                os << in << a << " += hd;\n";
                continue;
            }
            if (slot_rdx(p, s) || slot_rfma(p, s)) {
                os << in << a << " = fma(vd" << S << ", hd, " << a << ");\n";
                continue;
            }
            switch (p.slots[s].kind) {
                case S_CNT: os << in << a << " += h ? 1LL : 0LL;\n"; break;
                case S_NN: os << in << a << " += (h && sok" << S << ") ? 1LL : 0LL;\n"; break;
                case S_ISUM: os << in << a << " = (long long)((unsigned long long)" << a << " + (unsigned long long)((h && sok" << S
                                << ") ? sv" << S << " : 0LL));\n"; break;
                case S_IMIN: os << in << "if (h && sok" << S << " && sv" << S << " < " << a << ") " << a << " = sv" << S << ";\n"; break;
                case S_IMAX: os << in << "if (h && sok" << S << " && sv" << S << " > " << a << ") " << a << " = sv" << S << ";\n"; break;
                case S_FSUM: os << in << a << " += (h && sok" << S << ") ? sv" << S << " : 0.0;\n"; break;
                case S_FMIN: os << in << "if (h && sok" << S << " && sv" << S << " < " << a << ") " << a << " = sv" << S << ";\n"; break;
                case S_FMAX: os << in << "if (h && sok" << S << " && sv" << S << " > " << a << ") " << a << " = sv" << S << ";\n"; break;
            }
        }
        os << ind << "}\n";
    }
}

// Block reduction of the register accumulators into per-block partials.
// Where a register-path flush writes: the partial row index (the block in a
// plain launch, the unit's slot in a batch), the kind-table prefix and whether
// the staging arrays are carved from dynamic shared memory (batch bodies).
struct FlushCtx {
    std::string part_index = "blockIdx.x";
    std::string kinds = "P_";
    bool dyn_smem = false;
};

int regs_flush_smem(const Plan& p, int block) {
    int G = (int)p.domain;
    return (block / 32) * 8 * (std::max(G * p.nf, 1) + std::max(G * (p.ni + 1), 1));
}

void emit_regs_flush(std::ostringstream& os, const Plan& p, int block, const FlushCtx& fc = FlushCtx()) {
    int warps = block / 32;
    int G = (int)p.domain;
    int nf = p.nf, ni = p.ni;
    const int WF = std::max(G * nf, 1), WI = std::max(G * (ni + 1), 1);
    // the scan is done: let the dependent merge launch while blocks flush
    // (no effect when nothing was launched as a dependent)
    if (!fc.dyn_smem) os << "    asm volatile(\"griddepcontrol.launch_dependents;\");\n";
    // first-row keys and exact-double / shared accumulators back to the
    // variables (and types) the reduction below works on
    if (regs_fo_local(p))
        for (int g = 0; g < G; g++) os << "    long long fo" << g << " = vq_fo[" << g << "];\n";
    for (int g = 0; g < G; g++)
        for (size_t s = 0; s < p.slots.size(); s++) {
            if (!slot_rdx(p, s) && slot_alias(p, s) < 0) continue;
            if (p.slots[s].is_float()) os << "    double " << acc_name(p, g, (int)s) << " = " << acc_var(p, g, (int)s) << ";\n";
            else os << "    long long " << acc_name(p, g, (int)s) << " = (long long)" << acc_var(p, g, (int)s) << ";\n";
        }
    if (fc.dyn_smem) {
        os << "    __syncthreads();\n";
        os << "    double (*sh_f)[" << WF << "] = (double (*)[" << WF << "])vq_smem;\n";
        os << "    long long (*sh_i)[" << WI << "] = (long long (*)[" << WI << "])(vq_smem + " << warps * WF * 8 << ");\n";
    } else {
        os << "    __shared__ double sh_f[" << warps << "][" << WF << "];\n";
        os << "    __shared__ long long sh_i[" << warps << "][" << WI << "];\n";
    }
    os << "    const int fw = threadIdx.x >> 5;\n";
    for (int g = 0; g < G; g++) {
        for (size_t s = 0; s < p.slots.size(); s++) {
            std::string a = acc_name(p, g, (int)s);
            const char* op;
            switch (p.slots[s].kind) {
                case S_IMIN: op = "min"; break;
                case S_IMAX: op = "max"; break;
                case S_FMIN: op = "vq_fminr"; break;
                case S_FMAX: op = "vq_fmaxr"; break;
                default: op = nullptr; break;
            }
            os << "    for (int o = 16; o > 0; o >>= 1) { ";
            if (p.slots[s].is_float()) os << "double t = __shfl_xor_sync(0xffffffffu, " << a << ", o); ";
            else os << "long long t = __shfl_xor_sync(0xffffffffu, " << a << ", o); ";
            if (op) os << a << " = " << op << "(" << a << ", t); }\n";
            else if (p.slots[s].kind == S_ISUM) os << a << " = (long long)((unsigned long long)" << a << " + (unsigned long long)t); }\n";
            else os << a << " += t; }\n";
            int idx = p.slots[s].is_float() ? g * nf + p.slot_pos[s] : g * (ni + 1) + p.slot_pos[s];
            os << "    if ((threadIdx.x & 31) == 0) sh_" << (p.slots[s].is_float() ? "f" : "i") << "[fw][" << idx << "] = " << a << ";\n";
        }
        os << "    for (int o = 16; o > 0; o >>= 1) fo" << g << " = min(fo" << g << ", __shfl_xor_sync(0xffffffffu, fo" << g << ", o));\n";
        os << "    if ((threadIdx.x & 31) == 0) sh_i[fw][" << g * (ni + 1) + ni << "] = fo" << g << ";\n";
    }
    os << "    __syncthreads();\n";
    // merge folded into the scan (runs that pass the accumulators): the
    // block's combined partials go to the global accumulators as atomics; the
    // last block to arrive (threadfence before the arrival count, so every
    // earlier block's atomics are visible to it) reads each accumulator back
    // with an exchange that also restores its identity for the next run
    const bool fused = p.rfused && !fc.dyn_smem;
    if (fused) {
        // K copies of the accumulators, block b adding into copy b % K, so
        // the blocks that finish together spread their atomics over K times
        // the L2 lines; the last block folds the copies (exact integer adds,
        // or min / max)
        const int NF = std::max(nf, 1), NI1 = ni + 1, K = std::max(1, p.rcopies);
        os << "    if (P.racc_i) {\n";
        os << "        const int vq_cp = (int)(blockIdx.x % " << K << "u);\n";
        os << "        for (int t = threadIdx.x; t < " << G * nf << "; t += blockDim.x) {\n";
        os << "            const int s = t % " << NF << ";\n";
        os << "            double v = sh_f[0][t];\n";
        os << "            for (int w = 1; w < " << warps << "; w++) v = vq_fcomb(" << fc.kinds << "fkind(s), v, sh_f[w][t]);\n";
        os << "            vq_fx_add<true>(P.racc_fx + ((long long)vq_cp * " << G * nf << " + t) * 4, v, P.fx_lsb[s], P.racc_sp + t, P.error);\n";
        os << "        }\n";
        os << "        for (int t = threadIdx.x; t < " << G * NI1 << "; t += blockDim.x) {\n";
        os << "            const int s = t % " << NI1 << ";\n";
        os << "            long long v = sh_i[0][t];\n";
        os << "            for (int w = 1; w < " << warps << "; w++) v = vq_icomb(" << fc.kinds << "ikind(s), v, sh_i[w][t]);\n";
        os << "            vq_racc_add(P.racc_i + (long long)vq_cp * " << G * NI1 << " + t, " << fc.kinds << "ikind(s), v);\n";
        os << "        }\n";
        os << "        __threadfence();\n";
        os << "        __syncthreads();\n";
        os << "        __shared__ int vq_rlast;\n";
        os << "        if (threadIdx.x == 0) vq_rlast = atomicAdd(P.racc_done, 1u) == gridDim.x - 1u;\n";
        os << "        __syncthreads();\n";
        os << "        if (vq_rlast) {\n";
        os << "            __threadfence();\n";
        os << "            for (int t = threadIdx.x; t < " << G * nf << "; t += blockDim.x) {\n";
        os << "                vq_i64 c[4] = {0, 0, 0, 0};\n";
        os << "                for (int k = 0; k < " << K << "; k++)\n";
        os << "#pragma unroll\n";
        os << "                    for (int d = 0; d < 4; d++)\n";
        os << "                        c[d] = (vq_i64)((vq_u64)c[d] + atomicExch((unsigned long long*)(P.racc_fx + ((long long)k * " << G * nf
           << " + t) * 4 + d), 0ull));\n";
        os << "                P.rout_f[t] = vq_fx_result(c, P.fx_lsb[t % " << NF << "], atomicExch(P.racc_sp + t, 0u));\n";
        os << "            }\n";
        os << "            for (int t = threadIdx.x; t < " << G * NI1 << "; t += blockDim.x) {\n";
        os << "                const int kd = " << fc.kinds << "ikind(t % " << NI1 << ");\n";
        os << "                vq_i64 v = vq_racc_identity(kd);\n";
        os << "                for (int k = 0; k < " << K << "; k++)\n";
        os << "                    v = vq_icomb(kd, v, (vq_i64)atomicExch((unsigned long long*)(P.racc_i + (long long)k * " << G * NI1
           << " + t), (unsigned long long)vq_racc_identity(kd)));\n";
        os << "                P.rout_i[t] = (long long)v;\n";
        os << "            }\n";
        os << "            if (threadIdx.x == 0) {\n";
        os << "                *P.rerr_out = atomicExch(P.error, 0);\n";
        os << "                atomicExch(P.racc_done, 0u);\n";
        os << "            }\n";
        os << "        }\n";
        os << "    } else {\n";
    }
    // fixed-order combine over warps; kinds per bank entry
    os << "    for (int t = threadIdx.x; t < " << G * nf << "; t += blockDim.x) {\n";
    os << "        const int s = t % " << std::max(nf, 1) << ";\n";
    os << "        double v = sh_f[0][t];\n";
    os << "        for (int w = 1; w < " << warps << "; w++) v = vq_fcomb(" << fc.kinds << "fkind(s), v, sh_f[w][t]);\n";
    os << "        P.part_f[(long long)(" << fc.part_index << ") * " << G * nf << " + t] = v;\n    }\n";
    os << "    for (int t = threadIdx.x; t < " << G * (ni + 1) << "; t += blockDim.x) {\n";
    os << "        const int s = t % " << (ni + 1) << ";\n";
    os << "        long long v = sh_i[0][t];\n";
    os << "        for (int w = 1; w < " << warps << "; w++) v = vq_icomb(" << fc.kinds << "ikind(s), v, sh_i[w][t]);\n";
    os << "        P.part_i[(long long)(" << fc.part_index << ") * " << G * (ni + 1) << " + t] = v;\n    }\n";
    if (!fc.dyn_smem) {
        // merge by the last block to arrive (runs that pass P.mdone): the
        // partials are written above; a threadfence before the arrival count
        // makes them visible to the last block, whose warps each merge output
        // entries in block order, exactly as the merge kernel does
        const int tot = G * nf + G * (ni + 1), nfb = std::max(nf, 1);
        os << "    if (P.mdone) {\n";
        os << "        __threadfence();\n";
        os << "        __syncthreads();\n";
        os << "        __shared__ int vq_mlast;\n";
        os << "        if (threadIdx.x == 0) vq_mlast = atomicAdd(P.mdone, 1u) == gridDim.x - 1u;\n";
        os << "        __syncthreads();\n";
        os << "        if (vq_mlast) {\n";
        os << "            __threadfence();\n";
        os << "            for (int e = threadIdx.x >> 5; e < " << tot << "; e += blockDim.x >> 5)\n";
        os << "                merge_entry(e, P.part_f, P.part_i, (int)gridDim.x, " << G << ", " << nf << ", " << ni
           << ", P.mkinds, P.mkinds + " << nfb << ", P.mout_f, P.mout_i);\n";
        os << "            __syncthreads();\n";
        os << "            if (threadIdx.x == 0) {\n";
        os << "                *P.merr_out = atomicExch(P.error, 0);\n";
        os << "                atomicExch(P.mdone, 0u);\n";
        os << "            }\n";
        os << "        }\n";
        os << "    }\n";
    }
    if (fused) os << "    }\n";
}

// Atomic path: group table in global memory.
// gid_slot: the global join probe's group number (vq_gid) is the slot; the
// partitioned join, which has no build slots, inserts the packed key instead.
void emit_atomic_update(std::ostringstream& os, const Plan& p, const std::string& ind, const std::string& order,
                        bool gid_slot = false) {
    if (gid_slot) {
        os << ind << "const unsigned long long slot = vq_gid;\n";
    } else if (p.path == AggPath::Dense) {
        os << ind << "const unsigned long long slot = key;\n";
    } else {
        os << ind << "const unsigned long long slot = vq_insert(P.keys, P.cap_mask, P.cap, key, nullptr, P.error);\n";
        os << ind << "if (slot == VQ_NOSLOT) continue;\n";
    }
    os << ind << "const long long stride = (long long)P.cap + 1;\n";
    os << ind << "atomicMin(&P.first[slot], " << order << ");\n";
    for (size_t s = 0; s < p.slots.size(); s++) {
        std::string S = std::to_string(s);
        const Slot& sl = p.slots[s];
        int pos = p.slot_pos[s];
        std::string ai = "P.acc_i[" + std::to_string(pos) + " * stride + slot]";
        std::string aiu = "(unsigned long long*)&" + ai;
        switch (sl.kind) {
            case S_CNT: os << ind << "atomicAdd(" << aiu << ", 1ull);\n"; break;
            case S_NN: os << ind << "if (sok" << S << ") atomicAdd(" << aiu << ", 1ull);\n"; break;
            case S_ISUM: os << ind << "if (sok" << S << ") atomicAdd(" << aiu << ", (unsigned long long)sv" << S << ");\n"; break;
            case S_IMIN: os << ind << "if (sok" << S << ") atomicMin(&" << ai << ", sv" << S << ");\n"; break;
            case S_IMAX: os << ind << "if (sok" << S << ") atomicMax(&" << ai << ", sv" << S << ");\n"; break;
            case S_FMIN: os << ind << "if (sok" << S << " && !isnan(sv" << S << ")) atomicMin(" << aiu << ", vq_fkey(sv" << S << "));\n"; break;
            case S_FMAX: os << ind << "if (sok" << S << " && !isnan(sv" << S << ")) atomicMax(" << aiu << ", vq_fkey(sv" << S << "));\n"; break;
            case S_FSUM:
                os << ind << "if (sok" << S << ") vq_fx_add<true>(P.acc_fx + ((long long)" << pos << " * stride + (long long)slot) * 4, sv" << S
                   << ", P.fx_lsb[" << pos << "], P.special + (long long)" << pos << " * stride + slot, P.error);\n";
                break;
        }
    }
}

// Block-private shared-memory accumulators for the dense path: groups below
// smem_groups are updated with shared-memory atomics and flushed to the global
// table once per block; the layout is [first][int bank][fixed-point digits][flags].
struct CacheLayout {
    int C = 0;
    std::string first, ints, fx, sp;
};
// The cached group count is the launch-time value P.cache_n (vq_C in the
// generated code), so plans that differ only in domain share a kernel.
// Limb form (cache_limbs): the fixed-point region holds, per float sum, sixteen
// 32-bit limb counters a group (eight positive, eight negative; limb j of
// every group contiguous) instead of four 64-bit digit counters.
CacheLayout cache_layout(const Plan& p) {
    CacheLayout L;
    L.C = p.smem_groups;
    L.first = "((long long*)vq_smem)";
    L.ints = "(((long long*)vq_smem) + vq_C)";
    L.fx = "(((long long*)vq_smem) + (long long)vq_C * " + std::to_string(1 + p.ni) + ")";
    const int fx_longs = (p.cache_limbs ? 8 : 4) * p.nf;
    L.sp = "((unsigned*)(((long long*)vq_smem) + (long long)vq_C * " + std::to_string(1 + p.ni + fx_longs) + "))";
    return L;
}


// Opens "if (slot < C) { shared-memory update } else {" — the caller emits the
// global update and closes the brace.
void emit_cache_update(std::ostringstream& os, const Plan& p, const std::string& ind) {
    CacheLayout L = cache_layout(p);
    const std::string C = "vq_C";
    os << ind << "if (slot < (unsigned long long)vq_C) {\n";
    std::string in = ind + "    ";
    // MIN/MAX and first-row keys only ever move one way, so a plain read that
    // shows no improvement (possibly stale, never past the true value) skips
    // the atomic; most rows after the first few of a group skip it
    os << in << "if (ag_first < " << L.first << "[slot]) atomicMin(" << L.first << " + slot, ag_first);\n";
    for (size_t s = 0; s < p.slots.size(); s++) {
        std::string S = std::to_string(s), pos = std::to_string(p.slot_pos[s]);
        std::string ai = L.ints + " + " + pos + " * " + C + " + slot";
        std::string aiu = "(unsigned long long*)(" + ai + ")";
        switch (p.slots[s].kind) {
            case S_CNT:
            case S_NN:
                // a block's count stays below 2^32: a 32-bit add on the counter's low word
                if (p.cache_limbs && s == 0)  // the row count, read back: every 32,768 rows the group's limbs are normalised
                    os << in << "const unsigned vq_c0 = atomicAdd((unsigned*)(" << ai << "), (unsigned)ag" << S << ");\n";
                else if (p.cache_cnt32) os << in << "if (ag" << S << ") atomicAdd((unsigned*)(" << ai << "), (unsigned)ag" << S << ");\n";
                else os << in << "if (ag" << S << ") atomicAdd(" << aiu << ", (unsigned long long)ag" << S << ");\n";
                break;
            case S_ISUM:
                if (p.cache_fx32) os << in << "if (ah" << S << ") vq_add64_as32(" << ai << ", ag" << S << ");\n";
                else os << in << "if (ah" << S << ") atomicAdd(" << aiu << ", (unsigned long long)ag" << S << ");\n";
                break;
            case S_IMIN: os << in << "if (ah" << S << " && ag" << S << " < *(" << ai << ")) atomicMin(" << ai << ", ag" << S << ");\n"; break;
            case S_IMAX: os << in << "if (ah" << S << " && ag" << S << " > *(" << ai << ")) atomicMax(" << ai << ", ag" << S << ");\n"; break;
            case S_FMIN: os << in << "if (ah" << S << " && ag" << S << " < *" << aiu << ") atomicMin(" << aiu << ", ag" << S << ");\n"; break;
            case S_FMAX: os << in << "if (ah" << S << " && ag" << S << " > *" << aiu << ") atomicMax(" << aiu << ", ag" << S << ");\n"; break;
            case S_FSUM:
                if (p.cache_limbs) {
                    os << in << "if (ah" << S << ") { vq_limbs_add((unsigned*)" << L.fx << " + (long long)" << pos << " * 16 * " << C
                       << " + (long long)slot, " << C << ", fd" << S << "_0, fd" << S << "_1, fd" << S << "_2, fd" << S << "_3); if (fsp" << S
                       << ") atomicOr(" << L.sp << " + " << pos << " * " << C << " + slot, fsp" << S << "); }\n";
                    break;
                }
                os << in << "if (ah" << S << ") { " << (p.cache_fx32 ? "vq_fx_add_digits_s32(" : "vq_fx_add_digits_s(") << L.fx << " + (long long)" << pos << " * 4 * " << C
                   << " + (long long)slot, " << C << ", fd" << S << "_0, fd" << S << "_1, fd" << S << "_2, fd" << S << "_3); if (fsp" << S
                   << ") atomicOr(" << L.sp << " + " << pos << " * " << C << " + slot, fsp" << S << "); }\n";
                break;
        }
    }
    if (p.cache_limbs && p.nf > 0) {
        os << in << "if (((vq_c0 + (unsigned)ag0) >> 15) != (vq_c0 >> 15)) {\n";
        for (int f = 0; f < p.nf; f++)
            os << in << "    vq_limbs_norm((unsigned*)" << L.fx << " + (long long)" << f << " * 16 * " << C << " + (long long)slot, " << C << ");\n";
        os << in << "}\n";
    }
    os << ind << "} else {\n";
}

void emit_cache_init(std::ostringstream& os, const Plan& p, bool declare_smem = true) {
    CacheLayout L = cache_layout(p);
    const std::string C = "vq_C";
    if (declare_smem) os << "    extern __shared__ __align__(16) unsigned char vq_smem[];\n";
    os << "    const int vq_C = P.cache_n;\n";
    os << "    for (int i = threadIdx.x; i < " << C << "; i += blockDim.x) {\n";
    os << "        " << L.first << "[i] = 0x7FFFFFFFFFFFFFFFLL;\n";
    for (size_t s = 0; s < p.slots.size(); s++) {
        const Slot& sl = p.slots[s];
        if (sl.kind == S_FSUM) {
            std::string pos = std::to_string(p.slot_pos[s]);
            if (p.cache_limbs)
                os << "        for (int d = 0; d < 16; d++) ((unsigned*)" << L.fx << ")[(" << pos << " * 16 + d) * " << C << " + i] = 0u;\n";
            else
                os << "        for (int d = 0; d < 4; d++) " << L.fx << "[(" << pos << " * 4 + d) * " << C << " + i] = 0;\n";
            os << "        " << L.sp << "[" << pos << " * " << C << " + i] = 0u;\n";
            continue;
        }
        std::string init = "0LL";
        if (sl.kind == S_IMIN) init = "0x7FFFFFFFFFFFFFFFLL";
        if (sl.kind == S_IMAX) init = "(-0x7FFFFFFFFFFFFFFFLL - 1LL)";
        if (sl.kind == S_FMIN) init = "(long long)vq_fkey(1.7976931348623157e308)";
        if (sl.kind == S_FMAX) init = "(long long)vq_fkey(-1.7976931348623157e308)";
        os << "        " << L.ints << "[" << p.slot_pos[s] << " * " << C << " + i] = " << init << ";\n";
    }
    os << "    }\n    __syncthreads();\n";
}

void emit_cache_flush(std::ostringstream& os, const Plan& p) {
    CacheLayout L = cache_layout(p);
    const std::string C = "vq_C";
    os << "    __syncthreads();\n";
    os << "    for (int i = threadIdx.x; i < " << C << "; i += blockDim.x) {\n";
    os << "        if (" << L.ints << "[" << p.slot_pos[0] << " * " << C << " + i] == 0) continue;\n";
    os << "        const long long stride = (long long)P.cap + 1;\n";
    os << "        atomicMin(&P.first[i], " << L.first << "[i]);\n";
    for (size_t s = 0; s < p.slots.size(); s++) {
        int pos = p.slot_pos[s];
        std::string P_ = std::to_string(pos);
        std::string v = L.ints + "[" + P_ + " * " + C + " + i]";
        std::string g = "P.acc_i[" + P_ + " * stride + i]";
        switch (p.slots[s].kind) {
            case S_CNT:
            case S_NN:
            case S_ISUM: os << "        if (" << v << ") atomicAdd((unsigned long long*)&" << g << ", (unsigned long long)" << v << ");\n"; break;
            case S_IMIN: os << "        atomicMin(&" << g << ", " << v << ");\n"; break;
            case S_IMAX: os << "        atomicMax(&" << g << ", " << v << ");\n"; break;
            case S_FMIN: os << "        atomicMin((unsigned long long*)&" << g << ", (unsigned long long)" << v << ");\n"; break;
            case S_FMAX: os << "        atomicMax((unsigned long long*)&" << g << ", (unsigned long long)" << v << ");\n"; break;
            case S_FSUM:
                if (p.cache_limbs)
                    os << "        for (int d = 0; d < 4; d++) { const long long x = vq_limbs_digit((const unsigned*)" << L.fx << " + (long long)" << P_
                       << " * 16 * " << C << " + i, " << C << ", d); if (x) atomicAdd((unsigned long long*)&P.acc_fx[(" << P_
                       << " * stride + i) * 4 + d], (unsigned long long)x); }\n";
                else
                    os << "        for (int d = 0; d < 4; d++) { const long long x = " << L.fx << "[(" << P_ << " * 4 + d) * " << C
                       << " + i]; if (x) atomicAdd((unsigned long long*)&P.acc_fx[(" << P_ << " * stride + i) * 4 + d], (unsigned long long)x); }\n";
                os << "        if (" << L.sp << "[" << P_ << " * " << C << " + i]) atomicOr(&P.special[" << P_ << " * stride + i], "
                   << L.sp << "[" << P_ << " * " << C << " + i]);\n";
                break;
        }
    }
    os << "    }\n";
}

// Atomic path with warp aggregation: lanes whose rows fall into the same
// group (__match_any_sync peers) are reduced with redux.sync and only the
// lowest such lane updates the group table. Every reduction is exact and
// order-free: counts and integer sums wrap in 64 bits, MIN/MAX compare order
// keys, and float sums fold 128-bit fixed-point images of the values (the
// same integers the single-row update would add). When no two lanes of the
// warp share a group every lane updates its own row without reducing.
// Whether the dense path's hot-group registers are generated.
bool hot_on(const Plan& p) { return p.hot_n > 0 && p.path == AggPath::Dense && !p.is_join && !p.warp_agg; }

// One group's update from values in scope (slot, stride, ag_first, ag<s>,
// ah<s>, fd<s>_<k>, fsp<s>): the block's shared-memory cache when the slot is
// cached, else the global table.
void emit_lead_update(std::ostringstream& os, const Plan& p, const std::string& in3, bool cache) {
    if (cache) emit_cache_update(os, p, in3);
    // unguarded (fire-and-forget) MIN/MAX and first-row atomics: a read of the
    // current value to skip them measured slower on the global table (4M rows,
    // 65,536 Zipf groups mostly uncached: 118.9 against 74.8 us; 200K hash
    // keys: 201.6 against 197.7 us)
    os << in3 << "atomicMin(&P.first[slot], ag_first);\n";
    for (size_t s = 0; s < p.slots.size(); s++) {
        std::string S = std::to_string(s);
        int pos = p.slot_pos[s];
        std::string ai = "P.acc_i[" + std::to_string(pos) + " * stride + slot]";
        std::string aiu = "(unsigned long long*)&" + ai;
        switch (p.slots[s].kind) {
            case S_CNT:
            case S_NN: os << in3 << "if (ag" << S << ") atomicAdd(" << aiu << ", (unsigned long long)ag" << S << ");\n"; break;
            case S_ISUM: os << in3 << "if (ah" << S << ") atomicAdd(" << aiu << ", (unsigned long long)ag" << S << ");\n"; break;
            case S_IMIN: os << in3 << "if (ah" << S << ") atomicMin(&" << ai << ", ag" << S << ");\n"; break;
            case S_IMAX: os << in3 << "if (ah" << S << ") atomicMax(&" << ai << ", ag" << S << ");\n"; break;
            case S_FMIN: os << in3 << "if (ah" << S << ") atomicMin(" << aiu << ", ag" << S << ");\n"; break;
            case S_FMAX: os << in3 << "if (ah" << S << ") atomicMax(" << aiu << ", ag" << S << ");\n"; break;
            case S_FSUM:
                os << in3 << "if (ah" << S << ") { vq_fx_add_digits<true>(P.acc_fx + ((long long)" << pos << " * stride + (long long)slot) * 4, fd"
                   << S << "_0, fd" << S << "_1, fd" << S << "_2, fd" << S << "_3); if (fsp" << S << ") atomicOr(P.special + (long long)" << pos
                   << " * stride + slot, fsp" << S << "); }\n";
                break;
        }
    }
    if (cache) os << in3 << "}\n";  // closes the global branch opened by emit_cache_update
}

void emit_atomic_update_warp(std::ostringstream& os, const Plan& p, const std::string& ind, const std::string& order,
                             bool cache) {
    const std::string in = ind + "    ";
    os << ind << "unsigned long long slot = VQ_NOSLOT;\n";
    if (p.path == AggPath::Dense) os << ind << "if (live) slot = key;\n";
    else os << ind << "if (live) slot = vq_insert(P.keys, P.cap_mask, P.cap, key, nullptr, P.error);\n";
    os << ind << "live = live && slot != VQ_NOSLOT;\n";
    os << ind << "const unsigned act = __ballot_sync(0xffffffffu, live);\n";
    os << ind << "if (live) {\n";
    os << in << "const long long stride = (long long)P.cap + 1;\n";
    if (p.warp_agg) {
        os << in << "const unsigned peers = __match_any_sync(act, (unsigned)slot);\n";
        os << in << "const bool lead = (__ffs(peers) - 1) == lane;\n";
        os << in << "const bool solo = __all_sync(act, peers == (1u << lane));\n";
    } else {
        os << in << "const unsigned peers = 1u << lane; (void)act;\n";
        os << in << "const bool lead = true, solo = true;\n";
    }
    // per-lane fixed-point images of the float-sum inputs
    for (size_t s = 0; s < p.slots.size(); s++) {
        if (p.slots[s].kind != S_FSUM) continue;
        std::string S = std::to_string(s);
        os << in << "unsigned fw" << S << "[4], fs" << S << " = 0u; fw" << S << "[0] = fw" << S << "[1] = fw" << S << "[2] = fw" << S
           << "[3] = 0u;\n";
        os << in << "if (sok" << S << ") vq_fx_words(sv" << S << ", P.fx_lsb[" << p.slot_pos[s] << "], fw" << S << ", fs" << S
           << ", P.error);\n";
    }
    os << in << "long long ag_first;\n";
    for (size_t s = 0; s < p.slots.size(); s++) {
        std::string S = std::to_string(s);
        switch (p.slots[s].kind) {
            case S_CNT: case S_NN: os << in << "long long ag" << S << ";\n"; break;
            case S_ISUM: case S_IMIN: case S_IMAX: os << in << "long long ag" << S << "; bool ah" << S << ";\n"; break;
            case S_FMIN: case S_FMAX: os << in << "unsigned long long ag" << S << "; bool ah" << S << ";\n"; break;
            case S_FSUM:
                os << in << "long long fd" << S << "_0, fd" << S << "_1, fd" << S << "_2, fd" << S << "_3; unsigned fsp" << S << "; bool ah" << S
                   << ";\n";
                break;
        }
    }
    // single-row values
    os << in << "if (solo) {\n";
    std::string i2 = in + "    ";
    os << i2 << "ag_first = " << order << ";\n";
    for (size_t s = 0; s < p.slots.size(); s++) {
        std::string S = std::to_string(s);
        switch (p.slots[s].kind) {
            case S_CNT: os << i2 << "ag" << S << " = 1;\n"; break;
            case S_NN: os << i2 << "ag" << S << " = sok" << S << " ? 1 : 0;\n"; break;
            case S_ISUM: case S_IMIN: case S_IMAX: os << i2 << "ag" << S << " = sv" << S << "; ah" << S << " = sok" << S << ";\n"; break;
            case S_FMIN: case S_FMAX:
                os << i2 << "ah" << S << " = sok" << S << " && !isnan(sv" << S << "); ag" << S << " = vq_fkey(sv" << S << ");\n";
                break;
            case S_FSUM:
                os << i2 << "fd" << S << "_0 = fw" << S << "[0]; fd" << S << "_1 = fw" << S << "[1]; fd" << S << "_2 = fw" << S << "[2]; fd"
                   << S << "_3 = (long long)(int)fw" << S << "[3]; fsp" << S << " = fs" << S << "; ah" << S << " = sok" << S << ";\n";
                break;
        }
    }
    if (p.warp_agg) {
        // peer reductions
        os << in << "} else {\n";
        os << i2 << "ag_first = (long long)vq_wmin64(peers, (unsigned long long)(" << order << "));\n";
        for (size_t s = 0; s < p.slots.size(); s++) {
            std::string S = std::to_string(s);
            std::string any = "__ballot_sync(peers, sok" + S + ") != 0u";
            switch (p.slots[s].kind) {
                case S_CNT: os << i2 << "ag" << S << " = __popc(peers);\n"; break;
                case S_NN: os << i2 << "ag" << S << " = __popc(__ballot_sync(peers, sok" << S << "));\n"; break;
                case S_ISUM:
                    os << i2 << "ag" << S << " = (long long)vq_wsum64(peers, sok" << S << " ? (unsigned long long)sv" << S << " : 0ull); ah"
                       << S << " = " << any << ";\n";
                    break;
                case S_IMIN:
                    os << i2 << "ag" << S << " = (long long)(vq_wmin64(peers, (sok" << S << " ? (unsigned long long)sv" << S
                       << " : 0x7FFFFFFFFFFFFFFFull) ^ 0x8000000000000000ull) ^ 0x8000000000000000ull); ah" << S << " = " << any << ";\n";
                    break;
                case S_IMAX:
                    os << i2 << "ag" << S << " = (long long)(vq_wmax64(peers, (sok" << S << " ? (unsigned long long)sv" << S
                       << " : 0x8000000000000000ull) ^ 0x8000000000000000ull) ^ 0x8000000000000000ull); ah" << S << " = " << any << ";\n";
                    break;
                case S_FMIN:
                    os << i2 << "{ const bool o = sok" << S << " && !isnan(sv" << S << "); ag" << S << " = vq_wmin64(peers, o ? vq_fkey(sv" << S
                       << ") : 0xFFFFFFFFFFFFFFFFull); ah" << S << " = __ballot_sync(peers, o) != 0u; }\n";
                    break;
                case S_FMAX:
                    os << i2 << "{ const bool o = sok" << S << " && !isnan(sv" << S << "); ag" << S << " = vq_wmax64(peers, o ? vq_fkey(sv" << S
                       << ") : 0ull); ah" << S << " = __ballot_sync(peers, o) != 0u; }\n";
                    break;
                case S_FSUM:
                    os << i2 << "fd" << S << "_0 = vq_wsum32(peers, fw" << S << "[0]); fd" << S << "_1 = vq_wsum32(peers, fw" << S << "[1]); fd" << S
                       << "_2 = vq_wsum32(peers, fw" << S << "[2]);\n";
                    os << i2 << "fd" << S << "_3 = vq_wsum32(peers, fw" << S << "[3]) - ((long long)__popc(__ballot_sync(peers, (fw" << S
                       << "[3] >> 31) != 0u)) << 32);\n";
                    os << i2 << "fsp" << S << " = vq_redux_or(peers, fs" << S << "); ah" << S << " = " << any << ";\n";
                    break;
            }
        }
    }
    os << in << "}\n";
    if (hot_on(p)) {
        // the plan's hottest groups accumulate in this thread's registers
        os << in << "int vq_h = -1;\n";
        for (int h = 0; h < p.hot_n; h++)
            os << in << (h ? "else " : "") << "if (slot == P.hot[" << h << "]) vq_h = " << h << ";\n";
        os << in << "if (vq_h >= 0) {\n";
        os << in << "    switch (vq_h) {\n";
        for (int h = 0; h < p.hot_n; h++) {
            std::string H = std::to_string(h), i4 = in + "        ";
            os << in << "    case " << h << ": {\n";
            // a lane meets its rows in increasing order: its first row of the group holds the smallest order key
            os << i4 << "if (!hs" << H << ") { hs" << H << " = true; hf" << H << " = ag_first; }\n";
            for (size_t s = 0; s < p.slots.size(); s++) {
                std::string S = std::to_string(s), v = "hv" + H + "_" + S, hh = "hh" + H + "_" + S;
                switch (p.slots[s].kind) {
                    case S_CNT: case S_NN: os << i4 << v << " += ag" << S << ";\n"; break;
                    case S_ISUM:
                        os << i4 << "if (ah" << S << ") { " << v << " = (long long)((unsigned long long)" << v << " + (unsigned long long)ag" << S
                           << "); " << hh << " = true; }\n";
                        break;
                    case S_IMIN: case S_FMIN:
                        os << i4 << "if (ah" << S << " && ag" << S << " < " << v << ") " << v << " = ag" << S << "; " << hh << " = " << hh << " || ah" << S << ";\n";
                        break;
                    case S_IMAX: case S_FMAX:
                        os << i4 << "if (ah" << S << " && ag" << S << " > " << v << ") " << v << " = ag" << S << "; " << hh << " = " << hh << " || ah" << S << ";\n";
                        break;
                    case S_FSUM: {
                        std::string d = "hd" + H + "_" + S + "_";
                        os << i4 << "if (ah" << S << ") { " << d << "0 += fd" << S << "_0; " << d << "1 += fd" << S << "_1; " << d << "2 += fd" << S << "_2; "
                           << d << "3 += fd" << S << "_3; hp" << H << "_" << S << " |= fsp" << S << "; " << hh << " = true; }\n";
                        break;
                    }
                }
            }
            os << i4 << "break;\n" << in << "    }\n";
        }
        os << in << "    }\n" << in << "} else if (lead) {\n";
    } else {
        os << in << "if (lead) {\n";
    }
    emit_lead_update(os, p, in + "    ", cache);
    os << in << "}\n" << ind << "}\n";
}

// The dense path's hot groups: register accumulators (declared at kernel or
// body scope) and their flush into the cache or the table after the scan.
void emit_hot_decl(std::ostringstream& os, const Plan& p) {
    for (int h = 0; h < p.hot_n; h++) {
        std::string H = std::to_string(h);
        os << "    bool hs" << H << " = false; long long hf" << H << " = 0x7FFFFFFFFFFFFFFFLL;\n";
        for (size_t s = 0; s < p.slots.size(); s++) {
            std::string S = std::to_string(s), v = "hv" + H + "_" + S, hh = "bool hh" + H + "_" + S + " = false;";
            switch (p.slots[s].kind) {
                case S_CNT: case S_NN: os << "    long long " << v << " = 0;\n"; break;
                case S_ISUM: os << "    long long " << v << " = 0; " << hh << "\n"; break;
                case S_IMIN: os << "    long long " << v << " = 0x7FFFFFFFFFFFFFFFLL; " << hh << "\n"; break;
                case S_IMAX: os << "    long long " << v << " = (-0x7FFFFFFFFFFFFFFFLL - 1LL); " << hh << "\n"; break;
                case S_FMIN: os << "    unsigned long long " << v << " = 0xFFFFFFFFFFFFFFFFull; " << hh << "\n"; break;
                case S_FMAX: os << "    unsigned long long " << v << " = 0ull; " << hh << "\n"; break;
                case S_FSUM: {
                    std::string d = "hd" + H + "_" + S + "_";
                    os << "    long long " << d << "0 = 0, " << d << "1 = 0, " << d << "2 = 0, " << d << "3 = 0; unsigned hp" << H << "_" << S
                       << " = 0u; " << hh << "\n";
                    break;
                }
            }
        }
    }
}

void emit_hot_flush(std::ostringstream& os, const Plan& p, bool cache) {
    os << "    {\n        const long long stride = (long long)P.cap + 1;\n";
    for (int h = 0; h < p.hot_n; h++) {
        std::string H = std::to_string(h), in = "            ";
        os << "        if (hs" << H << ") {\n";
        os << in << "const unsigned long long slot = P.hot[" << h << "];\n";
        os << in << "const long long ag_first = hf" << H << ";\n";
        for (size_t s = 0; s < p.slots.size(); s++) {
            std::string S = std::to_string(s), v = "hv" + H + "_" + S, hh = "hh" + H + "_" + S;
            switch (p.slots[s].kind) {
                case S_CNT: case S_NN: os << in << "const long long ag" << S << " = " << v << ";\n"; break;
                case S_ISUM: case S_IMIN: case S_IMAX: os << in << "const long long ag" << S << " = " << v << "; const bool ah" << S << " = " << hh << ";\n"; break;
                case S_FMIN: case S_FMAX: os << in << "const unsigned long long ag" << S << " = " << v << "; const bool ah" << S << " = " << hh << ";\n"; break;
                case S_FSUM: {
                    std::string d = "hd" + H + "_" + S + "_";
                    os << in << "const long long fd" << S << "_0 = " << d << "0, fd" << S << "_1 = " << d << "1, fd" << S << "_2 = " << d << "2, fd" << S
                       << "_3 = " << d << "3; const unsigned fsp" << S << " = hp" << H << "_" << S << "; const bool ah" << S << " = " << hh << ";\n";
                    break;
                }
            }
        }
        emit_lead_update(os, p, in, cache);
        os << "        }\n";
    }
    os << "    }\n";
}

std::string kernel_head(const std::string& name, int block, int min_blocks = 0) {
    std::ostringstream os;
    os << "extern \"C\" __global__ void __launch_bounds__(" << block;
    if (min_blocks > 0) os << ", " << min_blocks;
    os << ") " << name
       << "(const __grid_constant__ VQParams P) {\n";
    return os.str();
}

// Chunk loop over the row segments: each warp takes 128-row chunks; lane l
// handles rows r0..r0+3 with 128-bit loads. The loop is software-pipelined:
// the loads of the warp's next chunk are issued before the current chunk is
// processed, so a warp keeps two chunks of column data in flight.
std::string seg_lookup(const std::string& c, const std::string& s0, const std::string& s1, const std::string& r0,
                       const std::string& lane_term = "lane * 4") {
    return "{ int lo = 0, hi = P.nseg - 1;\n"
           "          while (lo < hi) { const int mid = (lo + hi + 1) >> 1; if (P.seg[3 * mid + 2] <= " + c +
           ") lo = mid; else hi = mid - 1; }\n"
           "          " + s0 + " = P.seg[3 * lo]; " + s1 + " = P.seg[3 * lo + 1];\n"
           "          " + r0 + " = (" + s0 + " & ~127LL) + (" + c + " - P.seg[3 * lo + 2]) * 128 + " + lane_term + "; }\n";
}

void chunk_loop_open(std::ostringstream& os, const Plan& p, const Table* t, const std::set<int>& cols) {
    if (!p.pipeline) {
        os << "    const int lane = threadIdx.x & 31;\n"
              "    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;\n"
              "    for (long long c = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < P.nchunks; c += nw) {\n"
              "        long long s0 = 0, s1 = 0, r0 = 0;\n        " << seg_lookup("c", "s0", "s1", "r0");
        emit_loads(os, p, t, cols, "cv", "cm", "r0", "        ", true);
        return;
    }
    os << "    const int lane = threadIdx.x & 31;\n"
          "    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;\n"
          "    long long c = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;\n"
          "    long long s0 = 0, s1 = 0, r0 = 0;\n";
    emit_declare_regs(os, t, cols, "cv", "cm", "    ");
    os << "    if (c < P.nchunks) {\n        " << seg_lookup("c", "s0", "s1", "r0");
    emit_loads(os, p, t, cols, "cv", "cm", "r0", "        ", false);
    os << "    }\n";
    os << "    for (; c < P.nchunks; c += nw) {\n";
    os << "        const long long cn = c + nw;\n";
    os << "        long long ns0 = 0, ns1 = 0, nr0 = 0;\n";
    emit_declare_regs(os, t, cols, "nx", "nm", "        ");
    os << "        if (cn < P.nchunks) {\n        " << seg_lookup("cn", "ns0", "ns1", "nr0");
    emit_loads(os, p, t, cols, "nx", "nm", "nr0", "            ", false);
    os << "        }\n";
}

// ---- TMA-staged tile loop ---------------------------------------------------------------
// Each block walks tiles of T = warps × 128 rows. Thread 0 streams the tiles'
// column slices (and validity bitmaps) into a ring of S shared-memory stages
// with cp.async.bulk, each stage completing on its mbarrier; all warps read
// their 128-row slice from shared memory. A wait that does not complete within
// its poll limit raises error bit 8 and the whole block leaves the loop.
struct StageLayout {
    int T = 1024, S = 3, stage_bytes = 0, tx = 0;
    std::map<int, int> off, voff;
};

static int type_w(int t) {
    return (t == VEXQ_TYPE_INT64 || t == VEXQ_TYPE_FLOAT64) ? 8 : t == VEXQ_TYPE_BOOL ? 1 : 4;
}

StageLayout stage_layout(const Table* t, const std::set<int>& cols, int block, int budget) {
    StageLayout L;
    L.T = (block / 32) * 128;
    int o = 0;
    for (int c : cols) {
        L.off[c] = o;
        o += (L.T * type_w(t->cols[c].type) + 127) & ~127;
        L.tx += L.T * type_w(t->cols[c].type);
    }
    for (int c : cols) {
        if (!t->cols[c].nullable) continue;
        L.voff[c] = o;
        o += (L.T / 8 + 127) & ~127;
        L.tx += L.T / 8;
    }
    L.stage_bytes = std::max(o, 128);
    L.S = std::max(2, std::min(6, budget / L.stage_bytes));
    return L;
}

void emit_issue_fn(std::ostringstream& os, const Table* t, const std::set<int>& cols, const StageLayout& L,
                   const std::string& name) {
    os << "__device__ __forceinline__ void " << name
       << "(const VQParams& P, unsigned char* smem, unsigned long long* full, int stage, long long tile) {\n";
    os << "    int lo = 0, hi = P.nseg - 1;\n";
    os << "    while (lo < hi) { const int mid = (lo + hi + 1) >> 1; if (P.seg[3 * mid + 2] <= tile) lo = mid; else hi = mid - 1; }\n";
    os << "    const long long base = (P.seg[3 * lo] & ~" << (L.T - 1) << "LL) + (tile - P.seg[3 * lo + 2]) * " << L.T << ";\n";
    os << "    unsigned char* st = smem + stage * " << L.stage_bytes << ";\n";
    os << "    vq_mbar_expect_tx(full + stage, " << L.tx << "u);\n";
    for (int c : cols) {
        int w = type_w(t->cols[c].type);
        os << "    vq_bulk_g2s(st + " << L.off.at(c) << ", (const unsigned char*)P.col[" << c << "] + base * " << w << ", "
           << L.T * w << "u, full + stage);\n";
    }
    for (auto& kv : L.voff)
        os << "    vq_bulk_g2s(st + " << kv.second << ", P.valid[" << kv.first << "] + (base >> 3), " << L.T / 8
           << "u, full + stage);\n";
    os << "}\n";
}

void staged_loop_open(std::ostringstream& os, const Table* t, const std::set<int>& cols, const StageLayout& L,
                      const std::string& issue) {
    os << "    extern __shared__ __align__(128) unsigned char vq_smem[];\n";
    os << "    __shared__ __align__(8) unsigned long long vq_full[" << L.S << "];\n";
    os << "    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;\n";
    os << "    if (threadIdx.x == 0) {\n";
    os << "        for (int s = 0; s < " << L.S << "; s++) vq_mbar_init(&vq_full[s], 1u);\n";
    os << "        vq_fence_mbar_init();\n    }\n    __syncthreads();\n";
    os << "    if (threadIdx.x == 0)\n";
    os << "        for (int s = 0; s < " << L.S << "; s++) {\n";
    os << "            const long long tl = blockIdx.x + (long long)s * gridDim.x;\n";
    os << "            if (tl < P.nchunks) " << issue << "(P, vq_smem, vq_full, s, tl);\n        }\n";
    os << "    long long it = 0;\n    bool vq_timeout = false;\n";
    os << "    for (;; it++) {\n";
    os << "        const long long tile = blockIdx.x + it * gridDim.x;\n";
    os << "        if (tile >= P.nchunks) break;\n";
    os << "        const int stage = (int)(it % " << L.S << ");\n";
    os << "        const bool got = vq_mbar_wait(&vq_full[stage], (unsigned)((it / " << L.S << ") & 1), 1 << 20);\n";
    os << "        if (__syncthreads_or(!got)) { vq_timeout = true; break; }\n";
    os << "        long long s0, s1, r0;\n";
    os << "        { int lo = 0, hi = P.nseg - 1;\n";
    os << "          while (lo < hi) { const int mid = (lo + hi + 1) >> 1; if (P.seg[3 * mid + 2] <= tile) lo = mid; else hi = mid - 1; }\n";
    os << "          s0 = P.seg[3 * lo]; s1 = P.seg[3 * lo + 1];\n";
    os << "          r0 = (s0 & ~" << (L.T - 1) << "LL) + (tile - P.seg[3 * lo + 2]) * " << L.T << " + warp * 128 + lane * 4; }\n";
    os << "        const unsigned char* st = vq_smem + stage * " << L.stage_bytes << ";\n";
    os << "        const int so = warp * 128 + lane * 4;\n";
    for (int c : cols) {
        const Column& col = t->cols[c];
        std::string C = std::to_string(c);
        const char* ty = "unsigned";
        const char* fn = "vq_sld4_u32";
        switch (col.type) {
            case VEXQ_TYPE_INT64: ty = "long long"; fn = "vq_sld4_i64"; break;
            case VEXQ_TYPE_FLOAT64: ty = "double"; fn = "vq_sld4_f64"; break;
            case VEXQ_TYPE_DATE: ty = "int"; fn = "vq_sld4_i32"; break;
            case VEXQ_TYPE_BOOL: ty = "unsigned"; fn = "vq_sld4_u8"; break;
        }
        os << "        " << ty << " cv" << C << "[4]; " << fn << "(st + " << L.off.at(c) << ", so, cv" << C << ");\n";
        if (col.nullable) os << "        const unsigned cm" << C << " = vq_sbits4(st + " << L.voff.at(c) << ", so);\n";
    }
}

void staged_loop_close(std::ostringstream& os, const StageLayout& L, const std::string& issue) {
    os << "        __syncthreads();\n";
    os << "        if (threadIdx.x == 0) {\n";
    os << "            const long long nt = tile + (long long)" << L.S << " * gridDim.x;\n";
    os << "            if (nt < P.nchunks) { vq_fence_proxy_async(); " << issue << "(P, vq_smem, vq_full, stage, nt); }\n";
    os << "        }\n    }\n";
    // on a timeout: flag it, then wait (bounded) for the copies still in flight
    os << "    if (vq_timeout && threadIdx.x == 0) {\n";
    os << "        atomicOr(P.error, 8);\n";
    os << "        for (int k = 0; k < " << L.S << "; k++) {\n";
    os << "            const long long j = it + k, tl = blockIdx.x + j * gridDim.x;\n";
    os << "            if (tl < P.nchunks) vq_mbar_wait(&vq_full[j % " << L.S << "], (unsigned)((j / " << L.S << ") & 1), 1 << 20);\n";
    os << "        }\n    }\n";
}

// Closes the pipelined loop: the prefetched chunk becomes the current one.
void chunk_loop_close(std::ostringstream& os, const Plan& p, const Table* t, const std::set<int>& cols) {
    if (!p.pipeline) {
        os << "    }\n";
        return;
    }
    emit_copy_regs(os, t, cols, "        ");
    os << "        s0 = ns0; s1 = ns1; r0 = nr0;\n    }\n";
}


// ---- per-warp cp.async pipeline -------------------------------------------------------
// Each warp keeps `stages` 128-row chunk buffers in shared memory: while it
// computes chunk i from its buffer, the copies of the next stages-1 chunks are
// in flight, so bytes in flight do not cost registers. One commit group per
// iteration (possibly empty) keeps cp.async.wait_group's count exact.
struct AsyncLayout {
    int chunk_bytes = 0;
    std::map<int, int> off, voff;
};

AsyncLayout async_layout(const Table* t, const std::set<int>& cols) {
    AsyncLayout L;
    int o = 0;
    for (int c : cols) { L.off[c] = o; o += 128 * type_w(t->cols[c].type); }
    for (int c : cols)
        if (t->cols[c].nullable) { L.voff[c] = o; o += 16; }
    L.chunk_bytes = (o + 15) & ~15;
    return L;
}

void emit_async_issue_fn(std::ostringstream& os, const Table* t, const std::set<int>& cols, const AsyncLayout& L,
                         const std::string& name) {
    os << "__device__ __forceinline__ void " << name << "(const VQParams& P, unsigned char* dst, long long cc, int lane) {\n";
    os << "    int lo = 0, hi = P.nseg - 1;\n";
    os << "    while (lo < hi) { const int mid = (lo + hi + 1) >> 1; if (P.seg[3 * mid + 2] <= cc) lo = mid; else hi = mid - 1; }\n";
    os << "    const long long base = (P.seg[3 * lo] & ~127LL) + (cc - P.seg[3 * lo + 2]) * 128;\n";
    for (int c : cols) {
        const int w = type_w(t->cols[c].type);
        os << "    { const unsigned char* src = (const unsigned char*)P.col[" << c << "] + base * " << w << ";\n";
        os << "      for (int i = lane; i < " << 8 * w << "; i += 32) vq_cp16(dst + " << L.off.at(c) << " + i * 16, src + i * 16); }\n";
    }
    for (auto& kv : L.voff)
        os << "    if (lane == 0) vq_cp16(dst + " << kv.second << ", P.valid[" << kv.first << "] + (base >> 3));\n";
    os << "}\n";
}

// Lanes read the staged chunk strided: lane l takes rows l, l+32, l+64, l+96,
// each read from shared memory where it is used (consecutive lanes, consecutive
// words: no bank conflicts), so no register holds a row before its turn.
void async_loop_open(std::ostringstream& os, const Table* t, const std::set<int>& cols, const AsyncLayout& L, int stages,
                     const std::string& issue) {
    os << "    extern __shared__ __align__(16) unsigned char vq_abuf[];\n";
    os << "    const int lane = threadIdx.x & 31;\n";
    os << "    unsigned char* const wb = vq_abuf + (threadIdx.x >> 5) * " << stages * L.chunk_bytes << ";\n";
    os << "    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;\n";
    os << "    const long long c0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;\n";
    os << "    for (int s = 0; s < " << stages - 1 << "; s++) {\n";
    os << "        const long long cc = c0 + s * nw;\n";
    os << "        if (cc < P.nchunks) " << issue << "(P, wb + s * " << L.chunk_bytes << ", cc, lane);\n";
    os << "        vq_cp_commit();\n    }\n";
    os << "    long long it = 0;\n";
    os << "    for (long long c = c0; c < P.nchunks; c += nw, it++) {\n";
    os << "        const long long cn = c + " << stages - 1 << " * nw;\n";
    os << "        if (cn < P.nchunks) " << issue << "(P, wb + (int)((it + " << stages - 1 << ") % " << stages << ") * " << L.chunk_bytes
       << ", cn, lane);\n";
    os << "        vq_cp_commit();\n";
    os << "        vq_cp_wait<" << stages - 1 << ">();\n";
    os << "        __syncwarp();\n";
    os << "        const unsigned char* st = wb + (int)(it % " << stages << ") * " << L.chunk_bytes << ";\n";
    os << "        long long s0 = 0, s1 = 0, r0 = 0;\n        " << seg_lookup("c", "s0", "s1", "r0", "lane");
    for (int c : cols) {
        const Column& col = t->cols[c];
        std::string C = std::to_string(c);
        const char* ty = "unsigned";
        switch (col.type) {
            case VEXQ_TYPE_INT64: ty = "long long"; break;
            case VEXQ_TYPE_FLOAT64: ty = "double"; break;
            case VEXQ_TYPE_DATE: ty = "int"; break;
            case VEXQ_TYPE_BOOL: ty = "unsigned char"; break;
        }
        os << "        const " << ty << "* const cv" << C << " = (const " << ty << "*)(st + " << L.off.at(c) << ") + lane;\n";
        if (col.nullable) os << "        const unsigned cm" << C << " = vq_sbits4_strided(st + " << L.voff.at(c) << ", lane);\n";
    }
}

void async_loop_close(std::ostringstream& os) {
    os << "        __syncwarp();  // the buffer is refilled after every lane has read it\n";
    os << "    }\n";
    os << "    vq_cp_wait<0>();\n";
}

// Loop skeleton used by every scan kernel: TMA-staged tiles, the per-warp
// cp.async pipeline, or the (optionally register-prefetched) chunk loop.
struct ScanLoop {
    const Plan& p;
    const Table* t;
    std::set<int> cols;
    StageLayout L;
    AsyncLayout A;
    std::string issue;
    bool staged;
    int async_n = 0;
    int warps = 8;
    ScanLoop(const Plan& pp, const Table* tt, const std::set<int>& cc, int block, const std::string& name, bool allow_async = false)
        : p(pp), t(tt), cols(cc), staged(pp.staged) {
        int budget = pp.stage_budget > 0 ? pp.stage_budget : (block >= 256 ? 160 * 1024 : 96 * 1024);
        L = stage_layout(t, cols, block, budget);
        issue = "vq_issue_" + name;
        warps = block / 32;
        if (!staged && allow_async && pp.async_stages > 1) {
            async_n = pp.async_stages;
            A = async_layout(t, cols);
        }
    }
    int tile_rows() const { return staged ? L.T : 128; }
    // lane l holds rows l + 32k of a chunk (the cp.async pipeline) rather than 4l + k
    bool strided() const { return !staged && async_n > 0; }
    int smem() const { return staged ? L.S * L.stage_bytes : async_n ? warps * async_n * A.chunk_bytes : 0; }
    void prologue(std::ostringstream& os) const {
        if (staged) emit_issue_fn(os, t, cols, L, issue);
        else if (async_n) emit_async_issue_fn(os, t, cols, A, issue);
    }
    void open(std::ostringstream& os) const {
        if (staged) staged_loop_open(os, t, cols, L, issue);
        else if (async_n) async_loop_open(os, t, cols, A, async_n, issue);
        else chunk_loop_open(os, p, t, cols);
    }
    void close(std::ostringstream& os) const {
        if (staged) staged_loop_close(os, L, issue);
        else if (async_n) async_loop_close(os);
        else chunk_loop_close(os, p, t, cols);
    }
};

}  // namespace

int cache_group_bytes(const Plan& p) { return 8 + 8 * p.ni + (p.cache_limbs ? 68 : 36) * p.nf; }
int cache_bytes(const Plan& p) { return p.smem_groups * cache_group_bytes(p); }

static std::string gen_kind_tables(const Plan& p, const std::string& prefix = "P_");

// The four rows a lane holds in the current chunk: filter, project, aggregate.
static void emit_agg_rows(std::ostringstream& os, Plan& p, const std::vector<int>& key_nodes, bool cache,
                          bool strided = false) {
    os << "#pragma unroll\n        for (int k = 0; k < 4; k++) {\n";
    os << "            const long long r = r0 + " << (strided ? "(k << 5)" : "k") << ";\n";
    bool warp_sync = p.path != AggPath::Regs;  // atomic paths aggregate across the warp
    if (warp_sync) os << "            bool live = r >= s0 && r < s1;\n";
    else os << "            if (r < s0 || r >= s1) continue;\n";
    Gen g(p, os);
    if (strided) g.kidx = "(k << 5)";
    if (p.pred >= 0) {
        g.emit(p.pred);
        if (warp_sync) os << "            live = live && x" << p.pred << " && ok" << p.pred << ";\n";
        else os << "            if (!(x" << p.pred << " && ok" << p.pred << ")) continue;\n";
    }
    for (int k : key_nodes) g.emit(k);
    for (auto& s : p.slots) if (s.input >= 0) g.emit(s.input);
    emit_key(os, p, key_nodes, "            ");
    emit_slot_values(os, p, "            ", warp_sync ? "live" : "true");
    std::string order = order_expr(p, "r");
    if (p.path == AggPath::Regs) {
        if (p.regs_pred) emit_regs_update_pred(os, p, "            ", order);
        else emit_regs_update(os, p, "            ", order);
    } else {
        emit_atomic_update_warp(os, p, "            ", order, cache);
    }
    os << "        }\n";
}

// Generates the aggregate scan kernel (table → filter → project → aggregate).
static std::string gen_agg_kernel(Plan& p, const std::vector<int>& key_nodes, int block) {
    std::ostringstream os;
    std::set<int> cols;
    collect_cols(p, p.pred, cols);
    for (int k : key_nodes) collect_cols(p, k, cols);
    for (auto& s : p.slots) collect_cols(p, s.input, cols);
    // the cp.async pipeline owns the dynamic shared memory: register path only
    ScanLoop loop(p, p.t, cols, block, "agg", p.path == AggPath::Regs);
    p.tile = loop.tile_rows();
    p.smem = p.smem_groups > 0 ? cache_bytes(p) : loop.smem();
    loop.prologue(os);
    os << kernel_head("vq_agg", block, p.min_blocks);
    if (p.path == AggPath::Regs) emit_regs_decl(os, p);
    if (p.smem_groups > 0) emit_cache_init(os, p);
    if (hot_on(p)) emit_hot_decl(os, p);
    loop.open(os);
    emit_agg_rows(os, p, key_nodes, p.smem_groups > 0, loop.strided());
    loop.close(os);
    if (p.path == AggPath::Regs) emit_regs_flush(os, p, block);
    if (hot_on(p)) emit_hot_flush(os, p, p.smem_groups > 0);
    if (p.smem_groups > 0) emit_cache_flush(os, p);
    os << "}\n";
    return os.str();
}

// Batch body: one plan's aggregate scan over chunks [cbeg, cend), run by all
// warps of one block (warp w takes chunks cbeg+w, cbeg+w+warps, ...). The
// register path writes its partial row at pslot; the dense path always carries
// the shared-memory cache, sized at launch by P.cache_n (0 = none).
static std::string gen_agg_body(Plan& p, const std::string& name, int block) {
    std::ostringstream os;
    std::set<int> cols;
    collect_cols(p, p.pred, cols);
    for (int k : p.key_nodes) collect_cols(p, k, cols);
    for (auto& s : p.slots) collect_cols(p, s.input, cols);
    const bool cache = p.path == AggPath::Dense;  // sized at launch by P.cache_n (0 = none)
    if (p.path == AggPath::Regs) os << gen_kind_tables(p, name + "_");
    os << "__device__ __noinline__ void " << name
       << "(const VQParams& P, const long long cbeg, const long long cend, const long long pslot, unsigned char* vq_smem) {\n";
    if (p.path == AggPath::Regs) emit_regs_decl(os, p);
    if (cache) emit_cache_init(os, p, false);
    if (hot_on(p)) emit_hot_decl(os, p);
    os << "    const int lane = threadIdx.x & 31;\n";
    os << "    for (long long c = cbeg + (threadIdx.x >> 5); c < cend; c += " << block / 32 << ") {\n";
    os << "        long long s0 = 0, s1 = 0, r0 = 0;\n        " << seg_lookup("c", "s0", "s1", "r0");
    emit_loads(os, p, p.t, cols, "cv", "cm", "r0", "        ", true);
    emit_agg_rows(os, p, p.key_nodes, cache);
    os << "    }\n";
    if (p.path == AggPath::Regs) {
        FlushCtx fc;
        fc.part_index = "pslot";
        fc.kinds = name + "_";
        fc.dyn_smem = true;
        emit_regs_flush(os, p, block, fc);
    }
    if (hot_on(p)) emit_hot_flush(os, p, cache);
    if (cache) emit_cache_flush(os, p);
    os << "}\n";
    return os.str();
}

static void emit_direct_build_tail(std::ostringstream& os, bool block_claim);
static void emit_probe_rows(std::ostringstream& os, Plan& p, const std::vector<int>& key_nodes, bool strided);

// Batch body of a join's direct-mapped build over build chunks [cbeg, cend)
// (P: the build side's parameter block, mode 3): the build kernel's rows and
// tail, with the row and key counts added once per warp.
static std::string gen_build_body(Plan& p, const std::string& name, int block) {
    std::ostringstream os;
    std::set<int> cols;
    collect_cols(p, p.bpred, cols);
    collect_cols(p, p.bkey_node, cols);
    os << "__device__ __noinline__ void " << name
       << "(const VQParams& P, const long long cbeg, const long long cend, const long long pslot, unsigned char* vq_smem) {\n";
    os << "    const int lane = threadIdx.x & 31;\n";
    os << "    unsigned long long vq_nrows = 0ull;\n";
    os << "    unsigned vq_nk = 0u;\n";
    os << "    for (long long c = cbeg + (threadIdx.x >> 5); c < cend; c += " << block / 32 << ") {\n";
    os << "        long long s0 = 0, s1 = 0, r0 = 0;\n        " << seg_lookup("c", "s0", "s1", "r0");
    emit_loads(os, p, p.bt, cols, "cv", "cm", "r0", "        ", true);
    os << "        unsigned long long vq_d3[4] = {~0ull, ~0ull, ~0ull, ~0ull}, vq_k3[4];\n";
    os << "#pragma unroll\n        for (int k = 0; k < 4; k++) {\n";
    os << "            const long long r = r0 + k;\n";
    os << "            if (r < s0 || r >= s1) continue;\n";
    Gen g(p, os);
    if (p.bpred >= 0) {
        g.emit(p.bpred);
        os << "            if (!(x" << p.bpred << " && ok" << p.bpred << ")) continue;\n";
    }
    g.emit(p.bkey_node);
    const std::string K = std::to_string(p.bkey_node);
    os << "            if (!ok" << K << ") continue;  // NULL keys never join (exec/join.go:227-230)\n";
    os << "            const unsigned long long jk = (unsigned long long)(long long)x" << K << ";\n";
    os << "            const unsigned long long di = jk - (unsigned long long)P.dmin;\n";
    os << "            if (di >= P.drange) { atomicOr(P.error, 32); continue; }\n";
    os << "            vq_d3[k] = di;\n";
    os << "            vq_k3[k] = jk;\n";
    os << "        }\n";
    emit_direct_build_tail(os, false);
    os << "    }\n";
    os << "    for (int o = 16; o > 0; o >>= 1) {\n";
    os << "        vq_nrows += __shfl_xor_sync(0xffffffffu, vq_nrows, o);\n";
    os << "        vq_nk += __shfl_xor_sync(0xffffffffu, vq_nk, o);\n";
    os << "    }\n";
    os << "    if (lane == 0 && vq_nrows) atomicAdd(P.jtotal, vq_nrows);\n";
    os << "    if (lane == 0 && vq_nk) atomicAdd(P.jnkeys, (unsigned long long)vq_nk);\n";
    os << "}\n";
    return os.str();
}

// Batch body of a join's probe over probe chunks [cbeg, cend): the probe
// kernel's rows (direct-mapped table), folding into the plan's group table
// or, on the register path, into the unit's partial row at pslot.
static std::string gen_probe_body(Plan& p, const std::string& name, int block) {
    std::ostringstream os;
    std::set<int> cols;
    collect_cols(p, p.pred, cols);
    collect_cols(p, p.probe_key, cols);
    collect_cols(p, p.resid, cols);
    for (int k : p.key_nodes) collect_cols(p, k, cols);
    for (auto& s : p.slots) collect_cols(p, s.input, cols);
    if (p.path == AggPath::Regs) os << gen_kind_tables(p, name + "_");
    os << "__device__ __noinline__ void " << name
       << "(const VQParams& P, const long long cbeg, const long long cend, const long long pslot, unsigned char* vq_smem) {\n";
    if (p.path == AggPath::Regs) emit_regs_decl(os, p);
    os << "    const int lane = threadIdx.x & 31;\n";
    os << "    for (long long c = cbeg + (threadIdx.x >> 5); c < cend; c += " << block / 32 << ") {\n";
    os << "        long long s0 = 0, s1 = 0, r0 = 0;\n        " << seg_lookup("c", "s0", "s1", "r0");
    emit_loads(os, p, p.t, cols, "cv", "cm", "r0", "        ", true);
    emit_probe_rows(os, p, p.key_nodes, false);
    os << "    }\n";
    if (p.path == AggPath::Regs) {
        FlushCtx fc;
        fc.part_index = "pslot";
        fc.kinds = name + "_";
        fc.dyn_smem = true;
        emit_regs_flush(os, p, block, fc);
    }
    os << "}\n";
    return os.str();
}

std::string gen_batch_source(const std::vector<Plan*>& plans, int block, std::vector<int>& body_of, int& smem,
                             int& nbodies, bool build_role) {
    std::vector<std::string> bodies;
    std::map<std::string, int> index;
    body_of.clear();
    smem = 0;
    const std::string ph = "VQ_BODY_PLACEHOLDER";
    for (Plan* p : plans) {
        if (build_role && !p->is_join) fail(VEXQ_EINVAL, "a batched build body needs a join plan");
        std::string text;
        {
            // bodies cached per block size and role (aggregate or probe; build)
            std::lock_guard<std::mutex> lk(p->body_mu);
            const int key = block + (build_role ? (1 << 20) : 0);
            auto it = p->batch_body.find(key);
            if (it == p->batch_body.end())
                it = p->batch_body.emplace(key, build_role ? gen_build_body(*p, ph, block)
                                                : p->is_join ? gen_probe_body(*p, ph, block) : gen_agg_body(*p, ph, block)).first;
            text = it->second;
        }
        auto it = index.find(text);
        int b;
        if (it == index.end()) {
            b = (int)bodies.size();
            index[text] = b;
            bodies.push_back(text);
        } else {
            b = it->second;
        }
        body_of.push_back(b);
        if (p->path == AggPath::Regs) smem = std::max(smem, regs_flush_smem(*p, block));
    }
    // number the bodies in text order, so the same set of plan shapes gives the
    // same source (and one compiled module) whatever order the plans come in
    std::vector<int> order(bodies.size()), rank(bodies.size());
    std::iota(order.begin(), order.end(), 0);
    std::sort(order.begin(), order.end(), [&](int a, int c) { return bodies[a] < bodies[c]; });
    for (size_t r = 0; r < order.size(); r++) rank[order[r]] = (int)r;
    for (int& b : body_of) b = rank[b];
    std::vector<std::string> sorted(bodies.size());
    for (size_t b = 0; b < bodies.size(); b++) sorted[rank[b]] = bodies[b];
    bodies.swap(sorted);
    std::ostringstream os;
    os << prelude_source() << "\n";
    for (size_t b = 0; b < bodies.size(); b++) {
        std::string t = bodies[b], nm = "vq_body_" + std::to_string(b);
        for (size_t at = t.find(ph); at != std::string::npos; at = t.find(ph, at + nm.size())) t.replace(at, ph.size(), nm);
        os << t << "\n";
    }
    os << "extern \"C\" __global__ void __launch_bounds__(" << block << ") vq_batch(const __grid_constant__ VQBatchArgs A) {\n";
    os << "    extern __shared__ __align__(16) unsigned char vq_smem[];\n";
    os << "    __shared__ unsigned vq_unit;\n";
    os << "    for (;;) {\n";
    os << "        if (threadIdx.x == 0) vq_unit = atomicAdd(A.ticket, 1u);\n";
    os << "        __syncthreads();\n";
    os << "        const unsigned u = vq_unit;\n";
    os << "        __syncthreads();\n";
    os << "        if (u >= (unsigned)A.nunits) break;\n";
    os << "        const VQUnit U = A.units[u];\n";
    os << "        switch (U.body) {\n";
    for (size_t b = 0; b < bodies.size(); b++)
        os << "            case " << b << ": vq_body_" << b << "(A.params[U.plan], U.cbeg, U.cend, U.pslot, vq_smem); break;\n";
    os << "        }\n    }\n}\n";
    nbodies = (int)bodies.size();
    return os.str();
}

int dense_cache_groups(const Plan& p, int cache_kb) {
    if (p.path != AggPath::Dense || p.is_join || cache_kb <= 0) return 0;
    int per = cache_group_bytes(p);
    return (int)std::min<int64_t>(p.domain, (int64_t)cache_kb * 1024 / per);
}

// The direct-mapped build's chunk tail (vq_d3/vq_k3 hold the lane's four
// keys' table words and keys, ~0 where a row does not insert): four CAS in
// flight a lane, then their outcomes; with group numbers, one claim per warp
// and chunk (registers only: the lane's fresh rows are its four flags, in
// row order). Shared by the build kernel (mode 3) and the batched build body.
// block_claim (a chunk loop every warp of the block walks the same number of
// times): the warps' counts are summed in shared memory and the block takes
// its group numbers with one atomic per iteration instead of one per warp,
// the single counter every build row's claim serialises on; two buffers by
// iteration parity (vq_wsum, vq_gb, vq_par declared by the kernel) leave two
// barriers an iteration.
static void emit_direct_build_tail(std::ostringstream& os, bool block_claim) {
    os << "        if (P.mode == 3) {\n";
    os << "            unsigned long long vq_o3[4];\n";
    os << "#pragma unroll\n            for (int k = 0; k < 4; k++)\n";
    os << "                vq_o3[k] = vq_d3[k] != ~0ull ? atomicCAS(P.dmap + vq_d3[k], 0ull, (unsigned long long)(unsigned)(r0 + k) | 0xFFFFFFFF00000000ull) : 0ull;\n";
    os << "            bool vq_ok3[4];\n";
    os << "            int vq_n3 = 0;\n";
    os << "#pragma unroll\n            for (int k = 0; k < 4; k++) {\n";
    os << "                vq_ok3[k] = vq_d3[k] != ~0ull && vq_o3[k] == 0ull;\n";
    os << "                if (vq_d3[k] != ~0ull && vq_o3[k] != 0ull) atomicOr(P.error, 16);  // a repeated key: the general build runs\n";
    os << "                vq_n3 += vq_ok3[k] ? 1 : 0;\n";
    os << "            }\n";
    os << "            vq_nrows += (unsigned long long)vq_n3;\n";
    os << "            if (P.jgid) {\n";
    os << "                int inc = vq_n3;\n";
    os << "                for (int o = 1; o < 32; o <<= 1) { const int t = __shfl_up_sync(0xffffffffu, inc, o); if (lane >= o) inc += t; }\n";
    os << "                const int tot = __shfl_sync(0xffffffffu, inc, 31);\n";
    os << "                unsigned long long g = 0ull;\n";
    if (block_claim) {
        os << "                if (lane == 31) vq_wsum[vq_par][warp] = (unsigned)tot;\n";
        os << "                __syncthreads();\n";
        os << "                if (warp == 0) {\n";
        os << "                    const unsigned t = lane < (int)(blockDim.x >> 5) ? vq_wsum[vq_par][lane] : 0u;\n";
        os << "                    unsigned s = t;\n";
        os << "                    for (int o = 1; o < 32; o <<= 1) { const unsigned u = __shfl_up_sync(0xffffffffu, s, o); if (lane >= o) s += u; }\n";
        os << "                    unsigned long long b = 0ull;\n";
        os << "                    if (lane == 31 && s) b = atomicAdd(P.jnkeys, (unsigned long long)s);\n";
        os << "                    b = __shfl_sync(0xffffffffu, b, 31);\n";
        os << "                    if (lane < (int)(blockDim.x >> 5)) vq_wsum[vq_par][lane] = s - t;\n";
        os << "                    if (lane == 0) vq_gb[vq_par] = b;\n";
        os << "                }\n";
        os << "                __syncthreads();\n";
        os << "                g = vq_gb[vq_par] + (unsigned long long)vq_wsum[vq_par][warp] + (unsigned long long)(inc - vq_n3);\n";
        os << "                vq_par ^= 1;\n";
    } else {
        os << "                if (lane == 31 && tot) g = atomicAdd(P.jnkeys, (unsigned long long)tot);\n";
        os << "                g = __shfl_sync(0xffffffffu, g, 31) + (unsigned long long)(inc - vq_n3);\n";
    }
    os << "#pragma unroll\n                for (int k = 0; k < 4; k++) {\n";
    os << "                    if (!vq_ok3[k]) continue;\n";
    os << "                    P.dmap[vq_d3[k]] = (unsigned long long)(unsigned)(r0 + k) | ((unsigned long long)(unsigned)(~(int)g) << 32);\n";
    os << "                    P.jgkey[g] = (unsigned long long)((long long)vq_k3[k] - P.jgoff);\n";
    os << "                    g++;\n";
    os << "                }\n";
    os << "            } else {\n";
    os << "                vq_nk += (unsigned)vq_n3;\n";
    os << "            }\n";
    os << "        }\n";
}

// Join build kernel: filtered build rows with non-NULL keys are inserted into
// the build table (mode 0: insert + count, mode 1: place row ids).
static std::string gen_build_kernel(Plan& p, int key_node, int block) {
    std::ostringstream os;
    std::set<int> cols;
    collect_cols(p, p.bpred, cols);
    collect_cols(p, key_node, cols);
    ScanLoop loop(p, p.bt, cols, block, "build");
    p.btile = loop.tile_rows();
    p.bsmem = loop.smem();
    loop.prologue(os);
    os << kernel_head("vq_build", block);
    // distinct keys counted per lane and block, added to P.jnkeys once at the end
    os << "    __shared__ unsigned vq_nkeys;\n";
    os << "    unsigned long long vq_nrows = 0ull;\n";
    os << "    unsigned vq_nk = 0u;  // mode 2: fresh keys of this lane\n";
    os << "    if (threadIdx.x == 0) vq_nkeys = 0u;\n    __syncthreads();\n";
    // every warp of a block walks the same number of chunks (the TMA-staged
    // tile loop, or the plain chunk loop below with warps past the end idle),
    // so the direct build's group numbers are claimed once per block
    const bool block_claim = p.block_claim && (loop.staged || !p.pipeline);
    if (block_claim) os << "    __shared__ unsigned vq_wsum[2][32];\n    __shared__ unsigned long long vq_gb[2];\n    int vq_par = 0;\n";
    if (block_claim && !loop.staged) {
        os << "    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;\n";
        os << "    for (long long vb = (long long)blockIdx.x * (blockDim.x >> 5); vb < P.nchunks; vb += (long long)gridDim.x * (blockDim.x >> 5)) {\n";
        os << "        const long long c = vb + warp;\n";
        os << "        long long s0 = 0, s1 = 0, r0 = 0;\n";
        emit_declare_regs(os, p.bt, cols, "cv", "cm", "        ");
        os << "        if (c < P.nchunks) {\n            " << seg_lookup("c", "s0", "s1", "r0");
        emit_loads(os, p, p.bt, cols, "cv", "cm", "r0", "            ", false);
        os << "        }\n";
    } else {
        loop.open(os);
    }
    // mode 2 (keys unique in the last build): insert straight into the probe's
    // 16-byte slots; a lane's fresh slots wait in registers for their group
    // numbers, claimed once per warp and chunk
    os << "        long long vq_fs[4]; int vq_fr[4]; unsigned long long vq_fk[4]; int vq_nf = 0;\n";
    // mode 3: the lane's four table words, CAS'd together after the filter
    os << "        unsigned long long vq_d3[4] = {~0ull, ~0ull, ~0ull, ~0ull}, vq_k3[4];\n";
    os << "#pragma unroll\n        for (int k = 0; k < 4; k++) {\n";
    os << "            const long long r = r0 + k;\n";
    os << "            if (r < s0 || r >= s1) continue;\n";
    Gen g(p, os);
    if (p.bpred >= 0) {
        g.emit(p.bpred);
        os << "            if (!(x" << p.bpred << " && ok" << p.bpred << ")) continue;\n";
    }
    g.emit(key_node);
    std::string K = std::to_string(key_node);
    os << "            if (!ok" << K << ") continue;  // NULL keys never join (exec/join.go:227-230)\n";
    os << "            const unsigned long long jk = (unsigned long long)(long long)x" << K << ";\n";
    // mode 3 (keys unique and inside the dense range [dmin, dmin + drange)):
    // one CAS a row on the key's own word of the direct-mapped table
    os << "            if (P.mode == 3) {\n";
    os << "                const unsigned long long di = jk - (unsigned long long)P.dmin;\n";
    os << "                if (di >= P.drange) { atomicOr(P.error, 32); continue; }  // outside the range: the general build runs\n";
    os << "                vq_d3[k] = di;\n";
    os << "                vq_k3[k] = jk;\n";
    os << "            } else if (P.mode == 2) {\n";
    os << "                ulonglong2* sl = const_cast<ulonglong2*>(P.jslot);\n";
    os << "                long long at = -1;\n";
    os << "                if (jk == VQ_EMPTY_KEY) {\n";
    os << "                    const unsigned long long old = atomicCAS(&sl[P.jmask + 1].x, 0ull, 1ull);\n";
    os << "                    if (old == 0ull) at = (long long)P.jmask + 1; else atomicOr(P.error, 16);\n";
    os << "                } else {\n";
    os << "                    unsigned long long i = vq_hash(jk) & P.jmask;\n";
    os << "                    const unsigned long long lim = P.jmask < (unsigned long long)VQ_MAX_PROBES ? P.jmask + 1 : (unsigned long long)VQ_MAX_PROBES;\n";
    os << "                    unsigned long long n = 0;\n";
    os << "                    for (; n < lim; n++) {\n";
    os << "                        const unsigned long long old = atomicCAS(&sl[i].x, VQ_EMPTY_KEY, jk);\n";
    os << "                        if (old == VQ_EMPTY_KEY) { at = (long long)i; break; }\n";
    os << "                        if (old == jk) { atomicOr(P.error, 16); break; }  // a repeated key: the general build runs\n";
    os << "                        i = (i + 1) & P.jmask;\n";
    os << "                    }\n";
    os << "                    if (n == lim) atomicOr(P.error, 1);\n";
    os << "                }\n";
    os << "                if (at >= 0) {\n";
    os << "                    vq_nrows++;\n";
    os << "                    if (P.jgid) { vq_fs[vq_nf] = at; vq_fr[vq_nf] = (int)r; vq_fk[vq_nf] = at == (long long)P.jmask + 1 ? VQ_EMPTY_KEY : jk; vq_nf++; }\n";
    os << "                    else { sl[at].y = (unsigned long long)(unsigned)r | 0xFFFFFFFF00000000ull; vq_nk++; }\n";
    os << "                }\n";
    os << "            } else if (P.mode == 0) {\n";
    // pass 0 also keeps each slot's first row: a key with one build row needs
    // no row list, and a build whose keys never repeat skips pass 1
    os << "                bool fresh;\n";
    os << "                const unsigned long long js = vq_insert_fresh(P.jkeys, P.jmask, P.jmask + 1, jk, fresh, P.error);\n";
    os << "                if (js != VQ_NOSLOT) {\n";
    os << "                    atomicAdd(P.jcount + js, 1);\n";
    os << "                    vq_nrows++;\n";
    os << "                    if (fresh) { P.jfirst[js] = (int)r; vq_nk++; }\n";
    os << "                }\n";
    os << "            } else {\n";
    os << "                const unsigned long long js = vq_find(P.jkeys, P.jmask, P.jmask + 1, jk);\n";
    os << "                if (js != VQ_NOSLOT) P.jrows[P.jstart[js] + atomicAdd(P.jfill + js, 1)] = (int)r;\n";
    os << "            }\n";
    os << "        }\n";
    emit_direct_build_tail(os, block_claim);
    // mode 2 with group numbers (GROUP BY the join key): one claim per warp
    os << "        if (P.mode == 2 && P.jgid) {\n";
    os << "            int inc = vq_nf;\n";
    os << "            for (int o = 1; o < 32; o <<= 1) { const int t = __shfl_up_sync(0xffffffffu, inc, o); if (lane >= o) inc += t; }\n";
    os << "            const int tot = __shfl_sync(0xffffffffu, inc, 31);\n";
    os << "            unsigned long long base = 0ull;\n";
    os << "            if (lane == 31 && tot) base = atomicAdd(P.jnkeys, (unsigned long long)tot);\n";
    os << "            base = __shfl_sync(0xffffffffu, base, 31) + (unsigned long long)(inc - vq_nf);\n";
    os << "            ulonglong2* sl = const_cast<ulonglong2*>(P.jslot);\n";
    os << "            for (int j = 0; j < vq_nf; j++) {\n";
    os << "                const unsigned long long g = base + (unsigned long long)j;\n";
    os << "                const unsigned long long w = (unsigned long long)(unsigned)vq_fr[j] | ((unsigned long long)(unsigned)(~(int)g) << 32);\n";
    os << "                sl[vq_fs[j]].y = w;\n";
    os << "                P.jgkey[g] = (unsigned long long)((long long)vq_fk[j] - P.jgoff);\n";
    os << "            }\n";
    os << "        }\n";
    loop.close(os);
    // distinct keys a lane inserted, counted in registers (a shared counter
    // taking one atomic per fresh key serialised the warps)
    os << "    if (vq_nk) atomicAdd(&vq_nkeys, vq_nk);\n";
    os << "    __syncthreads();\n";
    os << "    if (threadIdx.x == 0 && vq_nkeys) atomicAdd(P.jnkeys, (unsigned long long)vq_nkeys);\n";
    os << "    for (int o = 16; o > 0; o >>= 1) vq_nrows += __shfl_xor_sync(0xffffffffu, vq_nrows, o);\n";
    os << "    if ((threadIdx.x & 31) == 0 && vq_nrows) atomicAdd(P.jtotal, vq_nrows);\n";
    os << "}\n";
    return os.str();
}

// One chunk of the join probe (a lane's four rows, loaded): a first pass runs
// the filter and the key and issues the four table loads, a second resolves
// them, runs the residual and folds every match into the aggregate in
// (probe row, chain position) order keys. Shared by the probe kernel and the
// batched probe body.
static void emit_probe_rows(std::ostringstream& os, Plan& p, const std::vector<int>& key_nodes, bool strided) {
    const std::string rk = std::string("r0 + ") + (strided ? "(k << 5)" : "k");
    std::string K = std::to_string(p.probe_key);
    // first pass over the lane's four rows: the filter, the key and the load
    // of the key's home slot, so four table loads are in flight at once
    os << "        unsigned long long vq_h[4]; ulonglong2 vq_s[4]; bool vq_on[4];\n";
    os << "#pragma unroll\n        for (int k = 0; k < 4; k++) {\n";
    os << "            const long long r = " << rk << ";\n";
    os << "            vq_on[k] = false;\n";
    os << "            if (r < s0 || r >= s1) continue;\n";
    {
        Gen g0(p, os);
        if (strided) g0.kidx = "(k << 5)";
        if (p.pred >= 0) {
            g0.emit(p.pred);
            os << "            if (!(x" << p.pred << " && ok" << p.pred << ")) continue;\n";
        }
        g0.emit(p.probe_key);
        os << "            if (!ok" << K << ") continue;\n";
        os << "            const unsigned long long jk = (unsigned long long)(long long)x" << K << ";\n";
        // direct-mapped table: the key's own word (0: no build row)
        os << "            if (P.dmap) {\n";
        os << "                const unsigned long long di = jk - (unsigned long long)P.dmin;\n";
        os << "                vq_s[k].y = di < P.drange ? vq_ld_dword(P.dmap + di) : 0ull;\n";
        os << "            } else {\n";
        os << "                vq_h[k] = jk == VQ_EMPTY_KEY ? P.jmask + 1 : (vq_hash(jk) & P.jmask);\n";
        os << "                vq_s[k] = vq_ld_slot(P.jslot + vq_h[k]);\n";
        os << "            }\n";
        os << "            vq_on[k] = true;\n";
    }
    os << "        }\n";
    os << "#pragma unroll\n        for (int k = 0; k < 4; k++) {\n";
    os << "            const long long r = " << rk << ";\n";
    os << "            if (!vq_on[k]) continue;\n";
    Gen g(p, os);
    if (strided) g.kidx = "(k << 5)";
    g.emit(p.probe_key);
    os << "            unsigned long long jc, jat = 0ull;\n";
    os << "            if (P.dmap) { jc = vq_s[k].y; if (jc == 0ull) continue; }\n";
    os << "            else if (!vq_find_slot_from(P.jslot, P.jmask, (unsigned long long)(long long)x" << K << ", vq_h[k], vq_s[k], jc, jat)) continue;\n";
    // a single-row chain carries its build row in the slot (count word ~group number, negative)
    os << "            const int ja = (int)(unsigned)jc, jn = (int)(jc >> 32);\n";
    if (p.join_gid) {
        os << "            const unsigned long long vq_gid = jn < 0 ? (unsigned long long)(unsigned)~jn : (unsigned long long)(unsigned)P.jgid[jat];\n";
        // the group table is sized by the last build's key count when the host
        // did not wait for this one: a number beyond it is raised, not written
        os << "            if (vq_gid >= P.cap) { atomicOr(P.error, 256); continue; }\n";
    }
    os << "            const int jb = jn < 0 ? 0 : ja, je = jn < 0 ? 1 : ja + jn;\n";
    os << "            for (int ji = jb; ji < je; ji++) {\n";
    os << "                const long long brow = jn < 0 ? (long long)ja : (long long)P.jrows[ji];\n";
    // above-join expressions: a fresh memo scope per match for build-side reads
    Gen g2(p, os);
    g2.done = g.done;
    g2.kidx = g.kidx;
    g2.ind = "                ";
    if (p.resid >= 0) {
        g2.emit(p.resid);
        os << "                if (!(x" << p.resid << " && ok" << p.resid << ")) continue;\n";
    }
    for (int k : key_nodes) g2.emit(k);
    for (auto& s : p.slots) if (s.input >= 0) g2.emit(s.input);
    emit_key(os, p, key_nodes, "                ");
    emit_slot_values(os, p, "                ");
    std::string order = order_expr(p, "((r << 16) | (long long)min(ji - jb, 65535))");
    if (p.path == AggPath::Regs) emit_regs_update(os, p, "                ", order);
    else emit_atomic_update(os, p, "                ", order, p.join_gid);
    os << "            }\n        }\n";
}

// Join probe kernel: probe rows pass the probe filter, look their key up, and
// every (build row, probe row) match runs the residual filter and is folded
// into the aggregate, in (probe row, chain position) order keys.
static std::string gen_probe_kernel(Plan& p, const std::vector<int>& key_nodes, int block) {
    std::ostringstream os;
    std::set<int> cols;
    collect_cols(p, p.pred, cols);
    collect_cols(p, p.probe_key, cols);
    collect_cols(p, p.resid, cols);
    for (int k : key_nodes) collect_cols(p, k, cols);
    for (auto& s : p.slots) collect_cols(p, s.input, cols);
    // the cp.async ring (register path only, where registers limit occupancy)
    ScanLoop loop(p, p.t, cols, block, "probe", p.path == AggPath::Regs);
    p.tile = loop.tile_rows();
    p.smem = loop.smem();
    loop.prologue(os);
    os << kernel_head("vq_agg", block, p.min_blocks);
    // a build the host did not wait for: its failure or emptiness is raised
    // in this kernel's error word, which comes back with the results
    os << "    if (P.berr && blockIdx.x == 0 && threadIdx.x == 0) {\n";
    os << "        const int be = *P.berr;\n";
    os << "        if (be & 8) atomicOr(P.error, 8);\n";
    os << "        if (be & ~8) atomicOr(P.error, 64);\n";
    os << "        else if (*P.bnk == 0ull) atomicOr(P.error, 128);\n";
    os << "    }\n";
    if (p.path == AggPath::Regs) emit_regs_decl(os, p);
    loop.open(os);
    emit_probe_rows(os, p, key_nodes, loop.strided());
    loop.close(os);
    if (p.path == AggPath::Regs) emit_regs_flush(os, p, block);
    os << "}\n";
    return os.str();
}

// ---- radix-partitioned join ----------------------------------------------------------
// Partition pass over one side (build: P.col = build table, its filter and key;
// probe: the probe table): rows that pass the filter with a non-NULL key go to
// partition = top pbits bits of the key hash. mode 0 counts rows per (block,
// partition) in a shared-memory histogram and stores it partition-major in
// P.phist; mode 1 re-runs the same rows in the same blocks and scatters
// (key, row) to the offsets the scan left in P.phist. Order inside a
// partition is not kept: the join pass sorts each build partition.
static std::string gen_part_kernel(Plan& p, const Table* t, int pred, int key_node, int block,
                                   const std::vector<int>& pay_cols = {}) {
    std::ostringstream os;
    std::set<int> cols;
    collect_cols(p, pred, cols);
    collect_cols(p, key_node, cols);
    for (int c : pay_cols) cols.insert(c);
    os << "extern \"C\" __global__ void __launch_bounds__(" << block << ") vq_part(const __grid_constant__ VQParams P) {\n";
    os << "    extern __shared__ __align__(16) unsigned vq_hist[];\n";
    os << "    const int np = P.nparts;\n";
    os << "    for (int i = threadIdx.x; i < np; i += blockDim.x)\n";
    os << "        vq_hist[i] = P.mode == 0 ? 0u : (unsigned)P.phist[(long long)i * gridDim.x + blockIdx.x];\n";
    os << "    __syncthreads();\n";
    // plain grid-stride chunk loop: both passes give every block the same rows
    os << "    const int lane = threadIdx.x & 31;\n"
          "    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;\n"
          "    for (long long c = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < P.nchunks; c += nw) {\n"
          "        long long s0 = 0, s1 = 0, r0 = 0;\n        " << seg_lookup("c", "s0", "s1", "r0");
    emit_loads(os, p, t, cols, "cv", "cm", "r0", "        ", true);
    os << "#pragma unroll\n        for (int k = 0; k < 4; k++) {\n";
    os << "            const long long r = r0 + k;\n";
    os << "            if (r < s0 || r >= s1) continue;\n";
    Gen g(p, os);
    if (pred >= 0) {
        g.emit(pred);
        os << "            if (!(x" << pred << " && ok" << pred << ")) continue;\n";
    }
    g.emit(key_node);
    std::string K = std::to_string(key_node);
    os << "            if (!ok" << K << ") continue;  // NULL keys never join (exec/join.go:227-230)\n";
    os << "            const unsigned long long jk = (unsigned long long)(long long)x" << K << ";\n";
    os << "            const unsigned part = (unsigned)(vq_hash(jk) >> (64 - P.pbits));\n";
    os << "            if (P.mode == 0) {\n";
    os << "                atomicAdd(vq_hist + part, 1u);\n";
    os << "            } else {\n";
    os << "                const unsigned pos = atomicAdd(vq_hist + part, 1u);\n";
    os << "                P.pkeys[pos] = jk;\n";
    os << "                P.prows[pos] = (int)r;\n";
    for (size_t j = 0; j < pay_cols.size(); j++) {
        const int c = pay_cols[j];
        const Column& col = t->cols[c];
        const std::string C = std::to_string(c), J = std::to_string(j);
        std::string w;
        switch (col.type) {
            case VEXQ_TYPE_FLOAT64: w = "(unsigned long long)__double_as_longlong(cv" + C + "[k])"; break;
            case VEXQ_TYPE_DATE: w = "(unsigned long long)(long long)cv" + C + "[k]"; break;
            default: w = "(unsigned long long)cv" + C + "[k]"; break;
        }
        os << "                P.qpay[" << J << "][pos] = " << w << ";\n";
        if (col.nullable) os << "                P.qpayv[" << J << "][pos] = (unsigned char)((cm" << C << " >> k) & 1u);\n";
    }
    os << "            }\n";
    os << "        }\n    }\n";
    os << "    __syncthreads();\n";
    os << "    if (P.mode == 0)\n";
    os << "        for (int i = threadIdx.x; i < np; i += blockDim.x) P.phist[(long long)i * gridDim.x + blockIdx.x] = (int)vq_hist[i];\n";
    os << "}\n";
    return os.str();
}

// Join pass: each block takes whole partitions. The partition's build entries
// (at most kRadixCap) are loaded into shared memory and bitonic-sorted by
// (key, build row), so equal keys form a run in build-row order, the chain
// order joinHashTable keeps (exec/join_table.go:496-517). Each probe entry
// binary-searches its run; every match runs the residual filter and is folded
// into the aggregate with order key (probe row << 16 | position in the run).
static const int kRadixCap = VQ_RADIX_CAP;
static const int kRadixMaxBits = VQ_RADIX_MAX_BITS;

// Partition-local aggregation (GROUP BY the join key): per build entry the
// accumulators of the group whose run starts there, in shared memory after the
// keys and rows: [first][int bank][fixed-point digits][flags] × rcap entries.
static int rlocal_bytes_per_entry(const Plan& p) { return 12 + 8 + 8 * p.ni + 36 * p.nf; }

static std::string gen_rjoin_kernel(Plan& p, const std::vector<int>& key_nodes, int block) {
    std::ostringstream os;
    const int cap = p.rcap;
    const std::string CAP = std::to_string(cap);
    os << "extern \"C\" __global__ void __launch_bounds__(" << block << ") vq_rjoin(const __grid_constant__ VQParams P) {\n";
    os << "    extern __shared__ __align__(16) unsigned char vq_sm[];\n";
    os << "    unsigned long long* sk = (unsigned long long*)vq_sm;\n";
    os << "    int* sr = (int*)(vq_sm + " << cap * 8 << ");\n";
    if (p.rlocal) {
        os << "    long long* LF = (long long*)(vq_sm + " << cap * 12 << ");\n";
        os << "    long long* LI = LF + " << cap << ";\n";
        os << "    long long* LX = LI + " << (long long)cap * p.ni << ";\n";
        os << "    unsigned* LS = (unsigned*)(LX + " << (long long)cap * 4 * p.nf << ");\n";
    }
    if (p.path == AggPath::Regs) emit_regs_decl(os, p);
    os << "    for (int part = blockIdx.x; part < P.nparts; part += gridDim.x) {\n";
    os << "        const long long b0 = P.bstart[part];\n";
    os << "        const int nb = (int)(P.bstart[part + 1] - b0);\n";
    os << "        int M = 1;\n        while (M < nb) M <<= 1;\n";
    os << "        __syncthreads();\n";
    os << "        for (int i = threadIdx.x; i < M; i += blockDim.x) {\n";
    os << "            if (i < nb) { sk[i] = P.bkeys[b0 + i]; sr[i] = P.brows[b0 + i]; }\n";
    os << "            else { sk[i] = 0xFFFFFFFFFFFFFFFFull; sr[i] = 0x7FFFFFFF; }  // pads sort after every entry\n";
    os << "        }\n";
    os << "        __syncthreads();\n";
    os << "        for (int kk = 2; kk <= M; kk <<= 1)\n";
    os << "            for (int j = kk >> 1; j > 0; j >>= 1) {\n";
    os << "                for (int i = threadIdx.x; i < M; i += blockDim.x) {\n";
    os << "                    const int ij = i ^ j;\n";
    os << "                    if (ij > i) {\n";
    os << "                        const unsigned long long ka = sk[i], kb = sk[ij];\n";
    os << "                        const int ra = sr[i], rb = sr[ij];\n";
    os << "                        const bool gt = ka > kb || (ka == kb && ra > rb);\n";
    os << "                        if (gt == ((i & kk) == 0)) { sk[i] = kb; sk[ij] = ka; sr[i] = rb; sr[ij] = ra; }\n";
    os << "                    }\n";
    os << "                }\n";
    os << "                __syncthreads();\n";
    os << "            }\n";
    if (p.rlocal) {  // identities for every entry's group accumulators
        std::vector<long long> iv = init_values(p);
        os << "        for (int i = threadIdx.x; i < nb; i += blockDim.x) {\n";
        os << "            LF[i] = 0x7FFFFFFFFFFFFFFFLL;\n";
        for (int s = 0; s < p.ni; s++) os << "            LI[" << s << " * " << CAP << " + i] = " << ilit(iv[s]) << ";\n";
        os << "            for (int d = 0; d < " << 4 * p.nf << "; d++) LX[(long long)i * " << 4 * p.nf << " + d] = 0;\n";
        for (int f = 0; f < p.nf; f++) os << "            LS[" << f << " * " << CAP << " + i] = 0u;\n";
        os << "        }\n        __syncthreads();\n";
    }
    os << "        const long long q1 = P.qstart[part + 1];\n";
    os << "        for (long long e = P.qstart[part] + threadIdx.x; e < q1; e += blockDim.x) {\n";
    os << "            const unsigned long long jkey = P.qkeys[e];\n";
    os << "            const long long r = P.qrows[e];\n";
    os << "            int lo = 0, hi = nb;\n";
    os << "            while (lo < hi) { const int mid = (lo + hi) >> 1; if (sk[mid] < jkey) lo = mid + 1; else hi = mid; }\n";
    os << "            for (int ji = lo; ji < nb && sk[ji] == jkey; ji++) {\n";
    os << "                const long long brow = sr[ji];\n";
    Gen g(p, os);
    g.gather = true;
    g.row = "r";
    g.ind = "                ";
    std::vector<int> pay_slot(p.t->cols.size(), -1);
    for (size_t j = 0; j < p.qpay_cols.size(); j++) pay_slot[p.qpay_cols[j]] = (int)j;
    g.pay_slot = &pay_slot;
    g.pay_row = "e";
    if (p.resid >= 0) {
        g.emit(p.resid);
        os << "                if (!(x" << p.resid << " && ok" << p.resid << ")) continue;\n";
    }
    for (int k : key_nodes) g.emit(k);
    for (auto& s : p.slots) if (s.input >= 0) g.emit(s.input);
    emit_key(os, p, key_nodes, "                ");
    emit_slot_values(os, p, "                ");
    std::string order = order_expr(p, "((r << 16) | (long long)min(ji - lo, 65535))");
    if (p.rlocal) {
        // the group is the key's run: shared-memory atomics on the run head `lo`
        const std::string in = "                ";
        os << in << "{ const long long ord = " << order << ";\n";
        os << in << "  if (ord < LF[lo]) atomicMin(LF + lo, ord);\n";
        for (size_t s = 0; s < p.slots.size(); s++) {
            const std::string S = std::to_string(s);
            const int pos = p.slot_pos[s];
            const std::string li = "LI + " + std::to_string(pos) + " * " + CAP + " + lo";
            switch (p.slots[s].kind) {
                // shared memory: 32-bit atomics (a partition's count stays below 2^32)
                case S_CNT: os << in << "  atomicAdd((unsigned*)(" << li << "), 1u);\n"; break;
                case S_NN: os << in << "  if (sok" << S << ") atomicAdd((unsigned*)(" << li << "), 1u);\n"; break;
                case S_ISUM: os << in << "  if (sok" << S << ") vq_add64_as32((long long*)(" << li << "), (long long)sv" << S << ");\n"; break;
                case S_IMIN: os << in << "  if (sok" << S << " && sv" << S << " < *(" << li << ")) atomicMin(" << li << ", sv" << S << ");\n"; break;
                case S_IMAX: os << in << "  if (sok" << S << " && sv" << S << " > *(" << li << ")) atomicMax(" << li << ", sv" << S << ");\n"; break;
                case S_FMIN:
                    os << in << "  if (sok" << S << " && !isnan(sv" << S << ")) { const unsigned long long q = vq_fkey(sv" << S
                       << "); if (q < *(unsigned long long*)(" << li << ")) atomicMin((unsigned long long*)(" << li << "), q); }\n";
                    break;
                case S_FMAX:
                    os << in << "  if (sok" << S << " && !isnan(sv" << S << ")) { const unsigned long long q = vq_fkey(sv" << S
                       << "); if (q > *(unsigned long long*)(" << li << ")) atomicMax((unsigned long long*)(" << li << "), q); }\n";
                    break;
                case S_FSUM:
                    os << in << "  if (sok" << S << ") vq_fx_add<true, true>(LX + ((long long)lo * " << p.nf << " + " << pos << ") * 4, sv" << S
                       << ", P.fx_lsb[" << pos << "], LS + " << pos << " * " << CAP << " + lo, P.error);\n";
                    break;
            }
        }
        os << in << "}\n";
    } else if (p.path == AggPath::Regs) {
        emit_regs_update(os, p, "                ", order);
    } else {
        emit_atomic_update(os, p, "                ", order);
    }
    os << "            }\n        }\n";
    if (p.rlocal) {
        // each group lives in one partition only: its totals go to the global
        // table with plain stores (the table starts at the identities)
        os << "        __syncthreads();\n";
        os << "        for (int i = threadIdx.x; i < nb; i += blockDim.x) {\n";
        os << "            if ((i > 0 && sk[i] == sk[i - 1]) || LI[" << p.slot_pos[0] << " * " << CAP << " + i] == 0) continue;\n";
        const int kn = key_nodes[0];
        const INode& kx = p.ir[kn];
        os << "            const bool ok" << kn << " = true;\n";
        os << "            const " << ctype(kx.type) << " x" << kn << " = (" << ctype(kx.type) << ")(long long)sk[i];\n";
        emit_key(os, p, key_nodes, "            ");
        if (p.path == AggPath::Dense) os << "            const unsigned long long slot = key;\n";
        else {
            os << "            const unsigned long long slot = vq_insert(P.keys, P.cap_mask, P.cap, key, nullptr, P.error);\n";
            os << "            if (slot == VQ_NOSLOT) continue;\n";
        }
        os << "            const long long stride = (long long)P.cap + 1;\n";
        os << "            P.first[slot] = LF[i];\n";
        for (int s = 0; s < p.ni; s++)
            os << "            P.acc_i[" << s << " * stride + slot] = LI[" << s << " * " << CAP << " + i];\n";
        for (int f = 0; f < p.nf; f++) {
            os << "            for (int d = 0; d < 4; d++) P.acc_fx[((long long)" << f << " * stride + slot) * 4 + d] = LX[((long long)i * "
               << p.nf << " + " << f << ") * 4 + d];\n";
            os << "            P.special[" << f << " * stride + slot] = LS[" << f << " * " << CAP << " + i];\n";
        }
        os << "        }\n";
    }
    os << "    }\n";
    if (p.path == AggPath::Regs) emit_regs_flush(os, p, block);
    os << "}\n";
    return os.str();
}

// Kind tables used by the register-path flush (per bank entry).
static std::string gen_kind_tables(const Plan& p, const std::string& prefix) {
    std::ostringstream os;
    std::vector<int> fk(std::max(p.nf, 1), 0), ik(p.ni + 1, 0);
    for (size_t s = 0; s < p.slots.size(); s++) {
        int k = p.slots[s].kind;
        int code = (k == S_IMIN || k == S_FMIN) ? 1 : (k == S_IMAX || k == S_FMAX) ? 2 : 0;
        if (p.slots[s].is_float()) fk[p.slot_pos[s]] = code;
        else ik[p.slot_pos[s]] = code;
    }
    ik[p.ni] = 1;  // first-occurrence key: min
    os << "__device__ __forceinline__ int " << prefix << "fkind(int s) { switch (s) {";
    for (size_t i = 0; i < fk.size(); i++) os << " case " << i << ": return " << fk[i] << ";";
    os << " } return 0; }\n";
    os << "__device__ __forceinline__ int " << prefix << "ikind(int s) { switch (s) {";
    for (size_t i = 0; i < ik.size(); i++) os << " case " << i << ": return " << ik[i] << ";";
    os << " } return 0; }\n";
    return os.str();
}

static const int kBlock = 256;

// Kernel tunables: the register path with many accumulators runs 128-thread
// blocks (more blocks per SM at ~200 registers a thread); VEXQ_TUNE
// ("block=128,pipeline=0") overrides for measurement sweeps.
static void choose_tunables(Plan& p) {
    int64_t acc = p.path == AggPath::Regs ? p.domain * (int64_t)(p.slots.size() + 1) : 0;
    p.block = acc > 24 ? 128 : 256;
    // dense group tables with the shared-memory cache: two 512-thread blocks
    // an SM (32 warps) hide the shared-atomic latency better than 256-thread
    // blocks at the same cache size (4M Zipf(1.1) rows: 46.1-48.2 / 69.6-76.8
    // us against 54.3-56.3 / 74.8 us at 1,000 / 65,536 groups)
    if (p.path == AggPath::Dense && !p.is_join) p.block = 512;
    // measured: software prefetch costs registers the register-accumulator path
    // needs (6M-row Q1: 74.9 µs without, 87.0 µs with); neutral for Q6
    // joins (measured, 6M-row probe): prefetch helps the register path and
    // costs the atomic path registers it needs for the table walk
    p.pipeline = p.is_join ? p.path == AggPath::Regs : p.path != AggPath::Regs;
    p.staged = false;  // measured: TMA staging is not faster for these scans yet
    p.regs_pred = true;
    // measured on Zipf(1.1) keys: per-lane shared-memory atomics beat folding
    // the peers of a warp first (the fold serialises over distinct groups)
    p.warp_agg = false;
    // dense path, shared-memory cache: 32-bit atomics (a 64-bit shared atomic
    // add measured 6x slower than a 32-bit one, 50x with a hot address). 4M
    // Zipf(1.1) rows, 1,000 / 65,536 groups: 60 / 75 us against 124 / 142 us
    // with 64-bit adds; the hottest groups in registers (hot=N) then cost more
    // than they save (67 / 82 us with one)
    p.cache_cnt32 = p.cache_fx32 = true;
    p.hot_n = 0;
    // float sums in the cache as 16-bit limbs with plain adds (no returned
    // value, no carry) instead of 32-bit word pairs whose carry comes back
    // from the returned old value: more atomics a row, measured slower (4M
    // Zipf rows, 1,000 / 65,536 groups: 54.2 / 79.1 against 48.2 / 76.8 us),
    // so a tunable (limbs=1)
    p.cache_limbs = false;
    // register path with many accumulators: three 128-thread blocks an SM
    // (~148 registers a thread), too few loads in flight to fill HBM; a
    // two-chunk cp.async pipeline a warp keeps the next chunk's columns in
    // flight without registers. 6M-row Q1 shape (6 groups x 8 accumulators):
    // 56.7 us against 59.8 us; with 40 warps an SM (one group) it costs
    // occupancy instead (Q6 shape: 43.9 us against 37.6 us). Join probes on
    // the register path likewise (Q12 shape, 1.5M x 6M rows: 0.269 against
    // 0.283 ms a query)
    p.async_stages = p.path == AggPath::Regs && acc > 24 ? 2 : 0;
    // measured: with the ring, one 384-thread block an SM (the same twelve
    // warps as three 128-thread blocks, a third of the partials) gave 63.2-63.7
    // against 64.2-65.1 us in one process and 67 against 63 us in the bench
    // loop; it stays a tunable (block=384)
    int cache_kb = 96;
    if (const char* e = std::getenv("VEXQ_TUNE")) {
        std::string s(e);
        auto get = [&](const char* k) -> int {
            size_t at = s.find(k);
            return at == std::string::npos ? -1 : std::atoi(s.c_str() + at + std::strlen(k));
        };
        int b = get("block="), pl = get("pipeline="), st = get("staged="), sb = get("stage_kb="), rp = get("regs_pred=");
        if (rp >= 0) p.regs_pred = rp != 0;
        int ck = get("cache_kb="), wa = get("warp_agg="), as = get("async="), mb = get("minb="), ho = get("hot=");
        int c32 = get("cnt32="), f32 = get("fx32="), gs = get("gsm="), cs = get("cs=");
        if (cs >= 0) p.stream_loads = cs != 0;
        const int kt = get("keep=");
        if (kt >= 0) p.keep_tables = kt != 0;
        const int fb = get("fastbuild=");
        if (fb >= 0) p.fast_build = fb != 0;
        const int dm = get("dmap=");
        if (dm >= 0) p.dmap_on = dm != 0;
        const int sp = get("spec=");
        if (sp >= 0) p.spec_on = sp != 0;
        const int bc = get("bclaim=");
        if (bc >= 0) p.block_claim = bc != 0;
        const int rc = get("rcopies=");
        if (rc >= 1 && rc <= 64) p.rcopies = rc;
        const int gr = get("graph=");
        if (gr == 0) p.graph_off = true;  // register-path runs as direct launches, not a replayed graph
        if (gs >= 0) p.grid_per_sm = gs;
        const int lb = get("limbs=");
        if (lb >= 0) p.cache_limbs = lb != 0;
        if (c32 >= 0) p.cache_cnt32 = c32 != 0;
        if (f32 >= 0) p.cache_fx32 = f32 != 0;
        if (ho >= 0 && p.path == AggPath::Dense && !p.is_join) p.hot_n = std::min(ho, VQ_MAXHOT);
        if (as >= 0) p.async_stages = as;
        if (mb >= 0) p.min_blocks = mb;
        if (ck >= 0) cache_kb = ck;
        if (wa >= 0) p.warp_agg = wa != 0;
        if (b == 64 || b == 128 || b == 256 || b == 384 || b == 512) p.block = b;
        const int ml = get("mlast=");
        if (ml >= 0) p.merge_last = ml != 0;
        if (pl >= 0) p.pipeline = pl != 0;
        if (st >= 0) p.staged = st != 0;
        if (sb > 0) p.stage_budget = sb * 1024;
    }
    // limbs take one row's canonical image at a time: not with warp folds or
    // the register hot groups, which add sums of several rows
    if (p.warp_agg || p.hot_n > 0) p.cache_limbs = false;
    p.smem_groups = 0;
    if (p.path == AggPath::Dense && !p.is_join && cache_kb > 0) {
        int per = cache_group_bytes(p);
        p.smem_groups = (int)std::min<int64_t>(p.domain, (int64_t)cache_kb * 1024 / per);
        p.staged = false;  // the cache owns the dynamic shared memory
    }
}

static void finish_compile(Plan& p, const std::vector<int>& key_nodes, bool join, int build_key_node) {
    p.key_nodes = key_nodes;
    p.bkey_node = build_key_node;
    p.range_epoch = p.t ? p.t->range_epoch : 0;
    p.brange_epoch = p.bt ? p.bt->range_epoch : 0;
    analyze(p);
    // large IN/LIKE code sets go to device bitsets; string rank tables beside them
    for (auto& n : p.ir) {
        if (n.k == NK::StrRank) {
            if ((int)p.sets.size() >= VQ_MAXSETS) fail(VEXQ_ENOTSUP, "too many large IN/LIKE sets and string MIN/MAX columns");
            n.set_idx = (int)p.sets.size();
            p.sets.push_back(n.rank.empty() ? std::vector<uint32_t>(1, 0u) : n.rank);
            continue;
        }
        if (n.k == NK::InCodes && n.codes.size() > 64) {
            if ((int)p.sets.size() >= VQ_MAXSETS) fail(VEXQ_ENOTSUP, "too many large IN/LIKE sets");
            std::vector<uint32_t> bits((n.codes.size() + 31) / 32, 0);
            for (size_t c = 0; c < n.codes.size(); c++) if (n.codes[c]) bits[c >> 5] |= 1u << (c & 31);
            n.set_idx = (int)p.sets.size();
            p.sets.push_back(std::move(bits));
        }
    }
    choose_path(p);
    p.join_gid = false;
    if (join && p.path != AggPath::Regs && p.keys.size() == 1 && !p.keys[0].nullable && p.keys[0].type == VEXQ_TYPE_INT64 &&
        std::getenv("VEXQ_NO_GID") == nullptr) {
        const KeyCol& k = p.keys[0];
        const bool jk = (k.build && k.col == p.build_key) || (!k.build && p.ir[p.probe_key].k == NK::Col && k.col == p.ir[p.probe_key].col);
        if (jk) {
            // hash-path key decoding (one key, shift 0): the group table's
            // key array holds the code the hash path would pack
            p.join_gid = true;
            p.path = AggPath::Hash;
            p.gid_koff = k.domain > 0 ? k.vmin : 0;
        }
    }
    choose_tunables(p);
    choose_regs_forms(p);
    choose_regs_fused(p);
    // numeric literals become launch-time values (first VQ_MAXLITS of them)
    p.lits.clear();
    for (auto& n : p.ir) {
        n.lit_slot = -1;
        if (n.k != NK::Lit || (int)p.lits.size() >= VQ_MAXLITS) continue;
        long long v;
        if (n.type == VEXQ_TYPE_INT64) v = n.li;
        else if (n.type == VEXQ_TYPE_DATE) v = n.ld;
        else if (n.type == VEXQ_TYPE_FLOAT64) std::memcpy(&v, &n.lf, 8);
        else continue;
        n.lit_slot = (int)p.lits.size();
        p.lits.push_back(v);
    }
    std::ostringstream src;
    if (p.stream_loads) src << "#define VQ_STREAM_LOADS 1\n";
    if (p.keep_tables) src << "#define VQ_KEEP_TABLES 1\n";
    src << prelude_source() << "\n" << gen_kind_tables(p) << "\n";
    std::string body = join ? gen_probe_kernel(p, key_nodes, p.block) : gen_agg_kernel(p, key_nodes, p.block);
    p.src_main = src.str() + body;
    if (join) {
        p.src_build = std::string(prelude_source()) + "\n" + gen_build_kernel(p, build_key_node, kBlock);
        p.src_part_b = std::string(prelude_source()) + "\n" + gen_part_kernel(p, p.bt, p.bpred, build_key_node, kBlock);
        // probe columns read above the join travel with the partitioned entries
        {
            std::set<int> above;
            std::function<void(int)> walk = [&](int i) {
                if (i < 0) return;
                const INode& n = p.ir[i];
                if (n.k == NK::Col && !n.build && n.tab == p.t) above.insert(n.col);
                for (int ch : n.ch) walk(ch);
            };
            walk(p.resid);
            for (int k : key_nodes) walk(k);
            for (auto& sl : p.slots) walk(sl.input);
            p.qpay_cols.clear();
            for (int c : above)
                if (p.qpay_cols.size() < 8) p.qpay_cols.push_back(c);
        }
        p.src_part_p = std::string(prelude_source()) + "\n" + gen_part_kernel(p, p.t, p.pred, p.probe_key, kBlock, p.qpay_cols);
        // GROUP BY exactly the join key on a group-table path: aggregate per partition
        p.rlocal = false;
        p.rcap = kRadixCap;
        if (p.path != AggPath::Regs && p.keys.size() == 1 && !p.keys[0].nullable) {
            const KeyCol& k = p.keys[0];
            const bool jk = (k.build && k.col == p.build_key) || (!k.build && k.col == p.ir[p.probe_key].col);
            const int per = rlocal_bytes_per_entry(p);
            int cap = kRadixCap;
            // ≤ 96 KB a block keeps two or more blocks per SM
            while (cap > 256 && (long long)cap * per > 96 * 1024) cap >>= 1;
            if (jk && (long long)cap * per <= 96 * 1024 && std::getenv("VEXQ_NO_RLOCAL") == nullptr) {
                p.rlocal = true;
                p.rcap = cap;
            }
        }
        p.src_rjoin = std::string(prelude_source()) + "\n" + gen_kind_tables(p) + "\n" + gen_rjoin_kernel(p, key_nodes, p.block);
    }
    std::ostringstream ex;
    ex << (join ? "join+agg" : "agg") << " path=" << (p.path == AggPath::Regs ? "regs" : p.path == AggPath::Dense ? "dense" : "hash")
       << " groups_domain=" << p.domain << " slots=" << p.slots.size() << " nf=" << p.nf << " ni=" << p.ni
       << " block=" << p.block
       << (p.staged ? " staged=tma" : (p.async_stages > 1 && p.path == AggPath::Regs) ? " async=" + std::to_string(p.async_stages)
           : p.pipeline ? " pipeline=1" : " pipeline=0")
       << (p.min_blocks > 0 ? " minb=" + std::to_string(p.min_blocks) : std::string())
       << " tile=" << p.tile << " smem=" << p.smem << " smem_groups=" << p.smem_groups << " warp_agg=" << p.warp_agg;
    if (hot_on(p)) ex << " hot_groups=" << p.hot_n;
    if (p.path == AggPath::Dense && !join && !(p.cache_cnt32 && p.cache_fx32)) ex << " atomics64";
    if (p.join_gid) ex << " groups=build_key_numbers";
    if (p.path == AggPath::Regs && !join) {
        int nx = 0, nm = 0, na = 0;
        for (size_t s = 0; s < p.slots.size(); s++) {
            nx += slot_rdx(p, s) && slot_alias(p, s) < 0;
            nm += slot_rfma(p, s);
            na += slot_alias(p, s) >= 0;
        }
        ex << " exact_int_sums=" << nx << " fma_sums=" << nm << " shared_sums=" << na;
        ex << " merge=" << (p.rfused ? "in_scan" : "kernel");
        if (p.rfused && p.rcopies > 1) ex << " rcopies=" << p.rcopies;
    }
    p.k_main = jit_get(p.src_main, "vq_agg", p.block, p.smem);
    ex << " regs=" << p.k_main.regs << " blocks_per_sm=" << p.k_main.max_blocks_per_sm;
    p.explain = ex.str();
    if (join) {
        p.k_build = jit_get(p.src_build, "vq_build", kBlock, p.bsmem);
        // radix-partitioned join (exec/parallel_join.go:72-109): the partition
        // histogram takes 4 bytes of shared memory per partition (set at launch)
        p.k_part_b = jit_get(p.src_part_b, "vq_part", kBlock, 4 << kRadixMaxBits);
        p.k_part_p = jit_get(p.src_part_p, "vq_part", kBlock, 4 << kRadixMaxBits);
        // 48 KB of keys and rows plus an opt-in margin for the register path's static staging
        p.k_rjoin = jit_get(p.src_rjoin, "vq_rjoin", p.block,
                            (p.rlocal ? p.rcap * rlocal_bytes_per_entry(p) : kRadixCap * 12) + 8192);
        p.radix = p.radix_bits != 0;
    }
    // device-side tables of the plan
    if (!p.sets.empty()) {
        size_t tot = 0;
        for (auto& s : p.sets) tot += s.size();
        p.d_sets.alloc(tot * 4);
        size_t off = 0;
        for (auto& s : p.sets) {
            h2d_now(p.d_sets.as<uint32_t>() + off, s.data(), s.size() * 4);
            off += s.size();
        }
    }
    auto upload_presence = [](const Table* tt, const std::vector<std::pair<int, int64_t>>& pl, DevBuf& dst) {
        if (pl.empty()) return;
        std::vector<uint8_t> pres(pl.size() * (size_t)tt->n_rg, 0);
        for (size_t i = 0; i < pl.size(); i++) {
            const Column& c = tt->cols[pl[i].first];
            for (int rg = 0; rg < tt->n_rg; rg++) pres[i * tt->n_rg + rg] = c.rg_present[rg][pl[i].second];
        }
        dst.alloc(pres.size());
        h2d_now(dst.p, pres.data(), pres.size());
    };
    upload_presence(p.t, p.presence, p.d_present);
    if (p.bt) upload_presence(p.bt, p.bpresence, p.d_bpresent);
}

static void copy_zone_tree(Plan& p, const vexq_expr* nodes, int nnodes, const int32_t* ch, int nch) {
    p.zn_nodes.assign(nodes, nodes + nnodes);
    p.zn_children.assign(ch, ch + nch);
    for (auto& n : p.zn_nodes) n.lit_str = nullptr;  // strings re-attached below
}

// Keeps string literals alive for the zone predicate (dates parse from them).
struct ZoneStrings {
    std::vector<std::string> s;
};
static std::map<const Plan*, ZoneStrings> g_zone_strings;
static std::mutex g_zone_mu;

static void keep_zone_strings(Plan& p, const vexq_expr* nodes, int nnodes) {
    std::lock_guard<std::mutex> lk(g_zone_mu);
    ZoneStrings& z = g_zone_strings[&p];
    z.s.resize(nnodes);
    for (int i = 0; i < nnodes; i++) {
        if (nodes[i].lit_str) {
            z.s[i] = nodes[i].lit_str;
            p.zn_nodes[i].lit_str = z.s[i].c_str();
        }
    }
}

Plan::~Plan() {
    {
        std::lock_guard<std::mutex> lk(g_zone_mu);
        g_zone_strings.erase(this);
    }
    if (rg_exec) cudaGraphExecDestroy(rg_exec);
    for (auto& e : ev)
        if (e) cudaEventDestroy(e);
    if (stream) cudaStreamDestroy(stream);
}

static void resolve_intkey(Plan& p) {
    // canUseIntKey (exec/agg_intkey.go:104-116): every GROUP BY column a dictionary string, ≤ 8 columns
    bool all_str = !p.keys.empty() && p.keys.size() <= 8;
    for (auto& k : p.keys) if (k.type != VEXQ_TYPE_STRING) all_str = false;
    p.intkey_order = all_str;
    size_t n = p.keys.size();
    p.intkey_width = n <= 2 ? 32 : n <= 4 ? 16 : 8;
}

Plan* compile_agg(Table* t, const vexq_agg_plan_desc* d) {
    if (!d || (d->naggs == 0 && d->ngroup_by == 0))
        fail(VEXQ_EINVAL, "exec: hash aggregate: no group-by columns or aggregate expressions");
    std::unique_ptr<Plan> p(new Plan);
    p->t = t;
    p->order = d->order;
    Translator tr{*p, d->nodes, d->nnodes, d->children, d->nchildren, t, nullptr};
    if (d->predicate >= 0) {
        p->pred = tr.tr(d->predicate);
        if (p->ir[p->pred].type != VEXQ_TYPE_BOOL) fail(VEXQ_EINVAL, "exec: filter predicate must return BOOL");
    }
    std::vector<int> key_nodes;
    for (int i = 0; i < d->ngroup_by; i++) {
        int c = d->group_by[i];
        if (c < 0 || c >= (int)t->cols.size()) fail(VEXQ_EINVAL, "GROUP BY column out of range");
        KeyCol k;
        k.col = c;
        k.build = false;
        k.name = t->cols[c].name;
        p->keys.push_back(k);
        INode n;
        n.k = NK::Col;
        n.col = c;
        n.tab = t;
        n.type = t->cols[c].type;
        n.nullable = t->cols[c].nullable;
        key_nodes.push_back(tr.add(n));
        p->gb_types.push_back(n.type);
    }
    std::vector<std::pair<int, int>> aggs;
    for (int j = 0; j < d->naggs; j++) aggs.push_back({d->aggs[j].kind, d->aggs[j].input >= 0 ? tr.tr(d->aggs[j].input) : -1});
    analyze(*p);
    plan_keys(*p);
    resolve_intkey(*p);
    plan_aggs(*p, aggs, d->aggs);
    // COUNT(DISTINCT) turns the integer-key path off (exec/aggregate.go:396-399):
    // groups keep plain first-row order
    if (p->ndist > 0) p->intkey_order = false;
    copy_zone_tree(*p, d->nodes, d->nnodes, d->children, d->nchildren);
    keep_zone_strings(*p, d->nodes, d->nnodes);
    p->zn_pred = d->predicate;
    finish_compile(*p, key_nodes, false, -1);
    return p.release();
}

Plan* compile_join(Table* bt, Table* pt, const vexq_join_plan_desc* d) {
    if (!d || (d->naggs == 0 && d->ngroup_by == 0))
        fail(VEXQ_EINVAL, "exec: hash aggregate: no group-by columns or aggregate expressions");
    std::unique_ptr<Plan> p(new Plan);
    p->is_join = true;
    p->t = pt;
    p->bt = bt;
    p->order = d->order;
    int nb = (int)bt->cols.size();
    if (d->build_key < 0 || d->build_key >= nb) fail(VEXQ_EINVAL, "exec: hash join: build key out of range");
    if (d->probe_key < 0 || d->probe_key >= (int)pt->cols.size()) fail(VEXQ_EINVAL, "exec: hash join: probe key out of range");
    int bkt = bt->cols[d->build_key].type, pkt = pt->cols[d->probe_key].type;
    if ((bkt != VEXQ_TYPE_INT64 && bkt != VEXQ_TYPE_DATE) || (pkt != VEXQ_TYPE_INT64 && pkt != VEXQ_TYPE_DATE))
        fail(VEXQ_ENOTSUP, "join keys must be INT64 or DATE columns on the GPU path");
    // build side predicate + key: scoped to the build table
    Translator tb{*p, d->nodes, d->nnodes, d->children, d->nchildren, bt, nullptr};
    tb.presence = &p->bpresence;
    if (d->build_predicate >= 0) {
        p->bpred = tb.tr(d->build_predicate);
        if (p->ir[p->bpred].type != VEXQ_TYPE_BOOL) fail(VEXQ_EINVAL, "exec: filter predicate must return BOOL");
    }
    INode bk;
    bk.k = NK::Col;
    bk.col = d->build_key;
    bk.tab = bt;
    bk.type = bkt;
    bk.nullable = bt->cols[d->build_key].nullable;
    int bkey = tb.add(bk);
    // probe side
    Translator tp{*p, d->nodes, d->nnodes, d->children, d->nchildren, pt, nullptr};
    tp.lit_strs = tb.lit_strs;
    if (d->probe_predicate >= 0) {
        p->pred = tp.tr(d->probe_predicate);
        if (p->ir[p->pred].type != VEXQ_TYPE_BOOL) fail(VEXQ_EINVAL, "exec: filter predicate must return BOOL");
    }
    INode pk;
    pk.k = NK::Col;
    pk.col = d->probe_key;
    pk.tab = pt;
    pk.type = pkt;
    pk.nullable = pt->cols[d->probe_key].nullable;
    p->probe_key = tp.add(pk);
    // above the join: joined schema (build columns, then probe columns)
    Translator ta{*p, d->nodes, d->nnodes, d->children, d->nchildren, pt, bt, nb, true};
    ta.lit_strs = tp.lit_strs;
    if (d->residual >= 0) {
        p->resid = ta.tr(d->residual);
        if (p->ir[p->resid].type != VEXQ_TYPE_BOOL) fail(VEXQ_EINVAL, "exec: filter predicate must return BOOL");
    }
    std::vector<int> key_nodes;
    for (int i = 0; i < d->ngroup_by; i++) {
        int c = d->group_by[i];
        if (c < 0 || c >= nb + (int)pt->cols.size()) fail(VEXQ_EINVAL, "GROUP BY column out of range");
        KeyCol k;
        k.build = c < nb;
        k.col = k.build ? c : c - nb;
        k.name = (k.build ? bt : pt)->cols[k.col].name;
        if (k.build && k.col == d->build_key && bkt == pkt && !bt->cols[k.col].nullable) {
            // equal to the probe key on every joined row: read it from the probe side
            // instead of gathering the build row
            k.build = false;
            k.col = d->probe_key;
            p->keys.push_back(k);
            key_nodes.push_back(p->probe_key);
            p->gb_types.push_back(bkt);
            continue;
        }
        p->keys.push_back(k);
        INode n;
        n.k = NK::Col;
        n.col = k.col;
        n.build = k.build;
        n.tab = k.build ? bt : pt;
        const Column& col = (k.build ? bt : pt)->cols[k.col];
        n.type = col.type;
        n.nullable = col.nullable;
        key_nodes.push_back(ta.add(n));
        p->gb_types.push_back(n.type);
    }
    std::vector<std::pair<int, int>> aggs;
    for (int j = 0; j < d->naggs; j++) aggs.push_back({d->aggs[j].kind, d->aggs[j].input >= 0 ? ta.tr(d->aggs[j].input) : -1});
    analyze(*p);
    plan_keys(*p);
    resolve_intkey(*p);
    plan_aggs(*p, aggs, d->aggs);
    if (p->ndist > 0) fail(VEXQ_ENOTSUP, "COUNT(DISTINCT) over a join is not supported on the GPU path");
    copy_zone_tree(*p, d->nodes, d->nnodes, d->children, d->nchildren);
    keep_zone_strings(*p, d->nodes, d->nnodes);
    p->zn_pred = d->probe_predicate;
    p->zn_bpred = d->build_predicate;
    p->radix_bits = d->radix_bits;
    p->build_key = d->build_key;
    finish_compile(*p, key_nodes, true, bkey);
    return p.release();
}

// Standalone filter (Filter.Next + BoolToSelVecInto, exec/filter.go:49-78):
// each lane evaluates four rows; warp ballots assemble a 128-row selection
// bitmap (bit = row passes: predicate true AND valid) per chunk.
// HAVING (planner/build.go:59-75, 512-637): exec.Filter over the
// aggregate's output batches, so the predicate is translated with the WHERE
// rules (coercion, StringEqExpr, casts) against the output schema — group-by
// columns, then aggregates — and evaluated per output row before ORDER BY /
// LIMIT; then only the first `visible` columns are kept (the hidden
// aggregates the planner appends for HAVING are projected away).
void gen_having_kernel(Plan& p);

void set_having(Plan& p, const vexq_expr* nodes, int nnodes, const int32_t* children, int nchildren, int root, int visible) {
    const int nout = (int)(p.keys.size() + p.outs.size());
    p.having_ir.clear();
    p.having_schema.reset();
    p.having_root = -1;
    p.having_visible = -1;
    if (root < 0) return;
    if (visible < -1 || visible > nout) fail(VEXQ_EINVAL, "HAVING keeps more columns than the aggregate outputs");
    if (!nodes || nnodes <= 0) fail(VEXQ_EINVAL, "HAVING without expression nodes");
    auto schema = std::make_unique<Table>();
    schema->cols.resize(nout);
    for (size_t k = 0; k < p.keys.size(); k++) {
        const KeyCol& kc = p.keys[k];
        Column& c = schema->cols[k];
        const Table* src = kc.build ? p.bt : p.t;
        c.name = kc.name.empty() ? src->cols[kc.col].name : kc.name;
        c.type = kc.type;
        c.nullable = true;
        c.per_rg_dicts = false;
        if (kc.type == VEXQ_TYPE_STRING) c.dict = src->cols[kc.col].dict;
    }
    for (size_t a = 0; a < p.outs.size(); a++) {
        Column& c = schema->cols[p.keys.size() + a];
        c.name = p.outs[a].name;
        c.type = p.outs[a].out_type;
        c.nullable = true;
        c.per_rg_dicts = false;
        if (p.outs[a].rank_dict) c.dict = *p.outs[a].rank_dict;
    }
    Plan hp;
    hp.t = schema.get();
    Translator tr{hp, nodes, nnodes, children, nchildren, schema.get(), nullptr};
    const int r = tr.tr(root);
    if (hp.ir[r].type != VEXQ_TYPE_BOOL) fail(VEXQ_EINVAL, "HAVING is not a boolean expression");
    p.having_ir = std::move(hp.ir);
    p.having_root = r;
    p.having_visible = visible;
    p.having_schema = std::move(schema);
    gen_having_kernel(p);
    const size_t at = p.explain.find(" having=");
    if (at != std::string::npos) p.explain.resize(at);
    p.explain += p.k_having.fn || !p.src_having.empty() ? " having=device" : " having=host";
}

// HAVING on the device, for plans whose groups live in a group table (dense,
// hash and join tables): vq_having runs one thread per compacted group, decodes
// the output columns the predicate reads exactly as the host result builder
// does (key columns from the packed key, COUNT, SUM, AVG = sum / non-null
// count, MIN/MAX, NULL when no input was non-null), evaluates the predicate
// with the scan kernels' expression code, and compacts the groups it keeps
// (one atomic a warp). Parameters, in the fields of VQParams:
//   in   P.keys / P.first / P.acc_i [NI][P.cap] / P.part_f [NF][P.cap], n = P.nchunks
//   out  P.pkeys / P.part_i / P.racc_i [NI][P.jmask] / P.rout_f [NF][P.jmask], count *P.jtotal
// Plans whose HAVING reads a string MIN/MAX output or a large IN set keep the
// host evaluation (k_having stays empty).
void gen_having_kernel(Plan& p) {
    p.k_having = JitKernel();
    p.src_having.clear();
    if (p.having_root < 0 || p.path == AggPath::Regs) return;
    const int nk = (int)p.keys.size();
    std::vector<INode> ir = p.having_ir;
    for (auto& n : ir) {
        n.lit_slot = -1;  // literals inline: the kernel is per plan
        if (n.k == NK::InCodes && n.codes.size() > 64) return;
        if (n.k == NK::StrRank || n.present_idx >= 0) return;
        if (n.k == NK::Col && n.col >= nk && p.outs[n.col - nk].rank_dict) return;
    }
    Plan hp;
    hp.ir = ir;
    std::ostringstream os;
    os << prelude_source() << "\n";
    os << kernel_head("vq_having", 256);
    os << "    const int lane = threadIdx.x & 31;\n";
    os << "    const long long vq_n = P.nchunks;\n";
    os << "    for (long long b0 = (long long)blockIdx.x * blockDim.x; b0 < vq_n; b0 += (long long)gridDim.x * blockDim.x) {\n";
    os << "        const long long j = b0 + threadIdx.x;\n";
    os << "        bool keep = false;\n";
    os << "        if (j < vq_n) {\n";
    os << "            const unsigned long long vq_key = P.keys[j];\n";
    const std::string in = "            ";
    Gen g(hp, os);
    g.ind = in;
    auto ival = [&](int slot) { return "P.acc_i[(long long)" + std::to_string(p.slot_pos[slot]) + " * P.cap + j]"; };
    auto fval = [&](int slot) {
        if (p.slots[slot].kind == S_FSUM) return "P.part_f[(long long)" + std::to_string(p.slot_pos[slot]) + " * P.cap + j]";
        return "vq_fkey_inv((unsigned long long)" + ival(slot) + ")";
    };
    for (size_t i = 0; i < ir.size(); i++) {
        const INode& n = ir[i];
        if (n.k != NK::Col) continue;
        const std::string x = "x" + std::to_string(i), ok = "ok" + std::to_string(i), ct = ctype(n.type);
        g.done[i] = 1;  // the output column is computed here, not read from a scanned column
        if (n.col < nk) {
            const KeyCol& k = p.keys[n.col];
            os << in << "long long kc" << i << "; bool kn" << i << " = false;\n";
            if (p.path != AggPath::Hash) {
                long long stride = 1;
                for (int kj = 0; kj < n.col; kj++) stride *= p.keys[kj].domain > 0 ? p.keys[kj].domain : 1;
                os << in << "kc" << i << " = (long long)((vq_key / " << stride << "ull) % " << k.domain << "ull);\n";
                if (k.nullable) os << in << "kn" << i << " = kc" << i << " == " << k.domain - 1 << "LL;\n";
            } else {
                const std::string m = k.bits >= 64 ? "0xFFFFFFFFFFFFFFFFull" : std::to_string((1ull << k.bits) - 1) + "ull";
                os << in << "{ const unsigned long long raw = (vq_key >> " << k.shift << ") & " << m << ";\n";
                if (k.domain > 0) {
                    os << in << "  kc" << i << " = (long long)raw;";
                    if (k.nullable) os << " kn" << i << " = kc" << i << " == " << k.domain - 1 << "LL;";
                    os << " }\n";
                } else if (k.type == VEXQ_TYPE_DATE) {
                    os << in << "  kn" << i << " = ((raw >> 32) & 1ull) != 0ull; kc" << i << " = (long long)(int)(unsigned)raw; }\n";
                } else {
                    os << in << "  kc" << i << " = (long long)raw; }\n";
                }
            }
            os << in << "const bool " << ok << " = !kn" << i << ";\n";
            std::string v = "kc" + std::to_string(i);
            if (k.domain > 0 && (k.type == VEXQ_TYPE_DATE || k.type == VEXQ_TYPE_INT64)) v = "(" + v + " + " + ilit(k.vmin) + ")";
            if (n.type == VEXQ_TYPE_BOOL) os << in << "const bool " << x << " = " << ok << " && " << v << " != 0LL;\n";
            else os << in << "const " << ct << " " << x << " = (" << ct << ")" << v << ";\n";
        } else {
            const AggOut& a = p.outs[n.col - nk];
            const Slot& sl = p.slots[a.value_slot];
            os << in << "const long long nn" << i << " = " << ival(a.nn_slot) << ";\n";
            if (a.kind == VEXQ_AGG_COUNT) {
                os << in << "const bool " << ok << " = true;\n";
                os << in << "const long long " << x << " = " << ival(a.value_slot) << ";\n";
                continue;
            }
            os << in << "const bool " << ok << " = nn" << i << " != 0LL;\n";
            if (a.kind == VEXQ_AGG_AVG)
                os << in << "const double " << x << " = " << ok << " ? " << fval(a.value_slot) << " / (double)nn" << i << " : 0.0;\n";
            else if (sl.is_float())
                os << in << "const double " << x << " = " << ok << " ? " << fval(a.value_slot) << " : 0.0;\n";
            else if (n.type == VEXQ_TYPE_BOOL)
                os << in << "const bool " << x << " = " << ok << " && " << ival(a.value_slot) << " != 0LL;\n";
            else
                os << in << "const " << ct << " " << x << " = " << ok << " ? (" << ct << ")" << ival(a.value_slot) << " : (" << ct << ")0;\n";
        }
    }
    g.emit(p.having_root);
    os << in << "keep = x" << p.having_root << " && ok" << p.having_root << ";\n";
    os << "        }\n";
    os << "        const unsigned bal = __ballot_sync(0xffffffffu, keep);\n";
    os << "        unsigned long long base = 0ull;\n";
    os << "        if (lane == 0 && bal) base = atomicAdd(P.jtotal, (unsigned long long)__popc(bal));\n";
    os << "        base = __shfl_sync(0xffffffffu, base, 0);\n";
    os << "        if (keep) {\n";
    os << "            const long long pos = (long long)(base + __popc(bal & ((1u << lane) - 1u)));\n";
    os << "            P.pkeys[pos] = P.keys[j];\n";
    os << "            P.part_i[pos] = P.first[j];\n";
    os << "            for (int s = 0; s < " << p.ni << "; s++) P.racc_i[(long long)s * (long long)P.jmask + pos] = P.acc_i[(long long)s * (long long)P.cap + j];\n";
    os << "            for (int f = 0; f < " << p.nf << "; f++) P.rout_f[(long long)f * (long long)P.jmask + pos] = P.part_f[(long long)f * (long long)P.cap + j];\n";
    os << "        }\n";
    os << "    }\n}\n";
    p.src_having = os.str();
    p.k_having = jit_get(p.src_having, "vq_having", 256, 0);
}

static void upload_scan_tables(Plan& p);

Plan* compile_filter(Table* t, const vexq_expr* nodes, int nnodes, const int32_t* children, int nchildren, int pred) {
    std::unique_ptr<Plan> p(new Plan);
    p->t = t;
    p->range_epoch = t->range_epoch;
    Translator tr{*p, nodes, nnodes, children, nchildren, t, nullptr};
    p->pred = tr.tr(pred);
    if (p->ir[p->pred].type != VEXQ_TYPE_BOOL) fail(VEXQ_EINVAL, "exec: filter predicate must return BOOL");
    analyze(*p);
    for (auto& n : p->ir) {
        if (n.k == NK::InCodes && n.codes.size() > 64) {
            if ((int)p->sets.size() >= VQ_MAXSETS) fail(VEXQ_ENOTSUP, "too many large IN/LIKE sets");
            std::vector<uint32_t> bits((n.codes.size() + 31) / 32, 0);
            for (size_t c = 0; c < n.codes.size(); c++) if (n.codes[c]) bits[c >> 5] |= 1u << (c & 31);
            n.set_idx = (int)p->sets.size();
            p->sets.push_back(std::move(bits));
        }
    }
    // the register chunk loop: the TMA stage ring (160 KB a block) would
    // leave one block per SM for a kernel that holds almost no state
    p->staged = false;
    p->pipeline = false;
    std::ostringstream os;
    std::set<int> cols;
    collect_cols(*p, p->pred, cols);
    ScanLoop loop(*p, t, cols, kBlock, "filter");
    p->tile = loop.tile_rows();
    p->smem = loop.smem();
    os << prelude_source() << "\n";
    loop.prologue(os);
    os << kernel_head("vq_filter", kBlock);
    // selected rows are counted in a register and added once per warp (one
    // global counter taking an atomic per bitmap word serialises the kernel)
    os << "    unsigned long long vq_cnt = 0ull;\n";
    loop.open(os);
    os << "        unsigned nib = 0u;\n";
    os << "#pragma unroll\n        for (int k = 0; k < 4; k++) {\n";
    os << "            const long long r = r0 + k;\n";
    os << "            if (r < s0 || r >= s1) continue;\n";
    Gen g(*p, os);
    g.emit(p->pred);
    os << "            if (x" << p->pred << " && ok" << p->pred << ") nib |= 1u << k;\n";
    os << "        }\n";
    // lane l holds rows base+4l..base+4l+3; word w of the chunk = lanes 8w..8w+7
    os << "        const unsigned long long spread = ((unsigned long long)nib) << (4 * (lane & 7));\n";
    os << "        unsigned word = (unsigned)spread;\n";
    os << "        for (int o = 1; o < 8; o <<= 1) word |= __shfl_xor_sync(0xffffffffu, word, o);\n";
    os << "        if ((lane & 7) == 0 && word) {\n";
    os << "            const long long wi = (r0 - lane * 4) / 32 + (lane >> 3);\n";
    os << "            atomicOr(reinterpret_cast<unsigned*>(P.acc_i) + wi, word);\n";
    os << "            vq_cnt += (unsigned long long)__popc(word);\n";
    os << "        }\n";
    loop.close(os);
    os << "    for (int o = 16; o > 0; o >>= 1) vq_cnt += __shfl_xor_sync(0xffffffffu, vq_cnt, o);\n";
    os << "    if ((threadIdx.x & 31) == 0 && vq_cnt) atomicAdd(P.ngroups, vq_cnt);\n";
    os << "}\n";
    p->src_main = os.str();
    p->k_main = jit_get(p->src_main, "vq_filter", kBlock, p->smem);
    upload_scan_tables(*p);
    p->explain = "filter";
    return p.release();
}

// Large IN sets and StringEqExpr presence rows of a one-table scan plan, to
// the device once.
static void upload_scan_tables(Plan& p) {
    const Table* t = p.t;
    if (!p.sets.empty()) {
        size_t tot = 0;
        for (auto& st : p.sets) tot += st.size();
        p.d_sets.alloc(tot * 4);
        size_t off = 0;
        for (auto& st : p.sets) {
            h2d_now(p.d_sets.as<uint32_t>() + off, st.data(), st.size() * 4);
            off += st.size();
        }
    }
    if (!p.presence.empty()) {
        std::vector<uint8_t> pres(p.presence.size() * (size_t)t->n_rg, 0);
        for (size_t i = 0; i < p.presence.size(); i++)
            for (int rg = 0; rg < t->n_rg; rg++)
                pres[i * t->n_rg + rg] = t->cols[p.presence[i].first].rg_present[rg][p.presence[i].second];
        p.d_present.alloc(pres.size());
        h2d_now(p.d_present.p, pres.data(), pres.size());
    }
}

// Filter → Project over one table (exec/filter.go:49-78, exec/project.go:64-128).
// Two generated kernels over the same chunk loop:
//   vq_pmark   the predicate's selection bitmap (bit r = row r kept; every
//              row of the scanned ranges when there is no predicate), words
//              assembled with warp shuffles, one atomicOr a word;
//   vq_pwrite  (projections only) for every kept row, its place in row order
//              (the chunk's offset from an exclusive scan of per-128-row-chunk
//              counts, plus the kept rows before it in its chunk) and the
//              projected values: raw 8-byte images into P.qpay[j % 8] and
//              validity bytes into P.qpayv[j % 8] for expressions j of the
//              group P.mode (eight expressions a launch).
Plan* compile_select(Table* t, const vexq_expr* nodes, int nnodes, const int32_t* children, int nchildren, int pred,
                     const int32_t* roots, int nroots) {
    if (nroots < 0 || nroots > 64) fail(VEXQ_EINVAL, "project: between 0 and 64 expressions");
    if (nroots > 0 && !roots) fail(VEXQ_EINVAL, "project: null expression roots");
    if (pred >= 0 && (!nodes || pred >= nnodes)) fail(VEXQ_EINVAL, "predicate index out of range");
    std::unique_ptr<Plan> p(new Plan);
    p->t = t;
    p->range_epoch = t->range_epoch;
    Translator tr{*p, nodes, nnodes, children, nchildren, t, nullptr};
    if (pred >= 0) {
        p->pred = tr.tr(pred);
        if (p->ir[p->pred].type != VEXQ_TYPE_BOOL) fail(VEXQ_EINVAL, "exec: filter predicate must return BOOL");
    }
    for (int j = 0; j < nroots; j++) {
        if (roots[j] < 0 || roots[j] >= nnodes) fail(VEXQ_EINVAL, "project: expression index out of range");
        const int r = tr.tr(roots[j]);
        const INode& n = p->ir[r];
        if (n.type == VEXQ_TYPE_STRING && n.k != NK::Col)
            fail(VEXQ_ENOTSUP, "project: a STRING expression must be a column reference");
        p->key_nodes.push_back(r);
    }
    analyze(*p);
    for (auto& n : p->ir) {
        if (n.k == NK::InCodes && n.codes.size() > 64) {
            if ((int)p->sets.size() >= VQ_MAXSETS) fail(VEXQ_ENOTSUP, "too many large IN/LIKE sets");
            std::vector<uint32_t> bits((n.codes.size() + 31) / 32, 0);
            for (size_t c = 0; c < n.codes.size(); c++) if (n.codes[c]) bits[c >> 5] |= 1u << (c & 31);
            n.set_idx = (int)p->sets.size();
            p->sets.push_back(std::move(bits));
        }
    }
    if (pred >= 0) {
        copy_zone_tree(*p, nodes, nnodes, children, nchildren);
        keep_zone_strings(*p, nodes, nnodes);
        p->zn_pred = pred;
    }
    p->staged = false;
    p->pipeline = false;
    std::set<int> pcols, wcols;
    if (p->pred >= 0) collect_cols(*p, p->pred, pcols);
    for (int r : p->key_nodes) collect_cols(*p, r, wcols);
    // the mark kernel
    {
        std::ostringstream os;
        ScanLoop loop(*p, t, pcols, kBlock, "pmark");
        p->tile = loop.tile_rows();
        p->smem = loop.smem();
        os << prelude_source() << "\n";
        loop.prologue(os);
        os << kernel_head("vq_pmark", kBlock);
        loop.open(os);
        os << "        unsigned nib = 0u;\n";
        os << "#pragma unroll\n        for (int k = 0; k < 4; k++) {\n";
        os << "            const long long r = r0 + k;\n";
        os << "            if (r < s0 || r >= s1) continue;\n";
        if (p->pred >= 0) {
            Gen g(*p, os);
            g.emit(p->pred);
            os << "            if (x" << p->pred << " && ok" << p->pred << ") nib |= 1u << k;\n";
        } else {
            os << "            nib |= 1u << k;\n";
        }
        os << "        }\n";
        os << "        const unsigned long long spread = ((unsigned long long)nib) << (4 * (lane & 7));\n";
        os << "        unsigned word = (unsigned)spread;\n";
        os << "        for (int o = 1; o < 8; o <<= 1) word |= __shfl_xor_sync(0xffffffffu, word, o);\n";
        os << "        if ((lane & 7) == 0 && word) atomicOr(reinterpret_cast<unsigned*>(P.acc_i) + (r0 - lane * 4) / 32 + (lane >> 3), word);\n";
        loop.close(os);
        os << "}\n";
        p->src_main = os.str();
        p->k_main = jit_get(p->src_main, "vq_pmark", kBlock, p->smem);
    }
    // the write kernel
    if (nroots > 0) {
        std::ostringstream os;
        ScanLoop loop(*p, t, wcols, kBlock, "pwrite");
        os << prelude_source() << "\n";
        loop.prologue(os);
        os << kernel_head("vq_pwrite", kBlock);
        loop.open(os);
        os << "        const unsigned* vq_w = reinterpret_cast<const unsigned*>(P.acc_i);\n";
        os << "#pragma unroll\n        for (int k = 0; k < 4; k++) {\n";
        os << "            const long long r = r0 + k;\n";
        os << "            if (r < s0 || r >= s1) continue;\n";
        os << "            const unsigned wv = vq_w[r >> 5];\n";
        os << "            if (!((wv >> (r & 31)) & 1u)) continue;\n";
        os << "            const long long cw = (r >> 7) << 2;\n";
        os << "            int below = __popc(wv & ((1u << (r & 31)) - 1u));\n";
        os << "            for (long long w = cw; w < (r >> 5); w++) below += __popc(vq_w[w]);\n";
        os << "            const long long pos = P.first[r >> 7] + below;\n";
        Gen g(*p, os);
        for (int j = 0; j < nroots; j++) {
            const int r = p->key_nodes[j];
            const INode& n = p->ir[r];
            os << "            if (P.mode == " << j / 8 << ") {\n";
            g.ind = "                ";
            std::fill(g.done.begin(), g.done.end(), 0);
            g.emit(r);
            std::string X = "x" + std::to_string(r), OK = "ok" + std::to_string(r), bits;
            switch (n.type) {
                case VEXQ_TYPE_FLOAT64: bits = "(unsigned long long)__double_as_longlong(" + X + ")"; break;
                case VEXQ_TYPE_INT64: bits = "(unsigned long long)" + X; break;
                case VEXQ_TYPE_DATE: bits = "(unsigned long long)(long long)" + X; break;
                case VEXQ_TYPE_STRING: bits = "(unsigned long long)" + X; break;
                default: bits = "(" + X + " ? 1ull : 0ull)"; break;
            }
            os << "                P.qpay[" << j % 8 << "][pos] = " << OK << " ? " << bits << " : 0ull;\n";
            os << "                P.qpayv[" << j % 8 << "][pos] = " << OK << " ? 1 : 0;\n";
            os << "            }\n";
        }
        os << "        }\n";
        loop.close(os);
        os << "}\n";
        p->src_build = os.str();
        p->k_build = jit_get(p->src_build, "vq_pwrite", kBlock, 0);
    }
    upload_scan_tables(*p);
    p->explain = nroots ? "project" : "filter";
    return p.release();
}

// ---- zone maps (planner/physical.go:624-750) ----------------------------------------------------

static bool literal_int64(const vexq_expr& e, int64_t* v, int* lk) {
    if (e.kind != VEXQ_E_LITERAL) return false;
    *lk = e.lit_kind;
    if (e.lit_kind == VEXQ_LIT_INT) { *v = e.lit_int; return true; }
    if (e.lit_kind == VEXQ_LIT_FLOAT) { std::memcpy(v, &e.lit_float, 8); return true; }
    if (e.lit_kind == VEXQ_LIT_STRING) return parse_date(e.lit_str, v);
    return false;
}

static bool zone_rec(const Plan& p, int idx, const Table& t, int rg) {
    if (idx < 0 || idx >= (int)p.zn_nodes.size()) return true;
    const vexq_expr& e = p.zn_nodes[idx];
    auto ch = [&](int k) { return p.zn_children[e.child0 + k]; };
    if (e.kind == VEXQ_E_AND) {
        for (int k = 0; k < e.nchildren; k++) if (!zone_rec(p, ch(k), t, rg)) return false;
        return true;
    }
    if (e.kind == VEXQ_E_OR) {
        if (e.nchildren == 0) return true;
        for (int k = 0; k < e.nchildren; k++) if (zone_rec(p, ch(k), t, rg)) return true;
        return false;
    }
    if (e.kind == VEXQ_E_BETWEEN) {
        const vexq_expr& c = p.zn_nodes[ch(0)];
        if (c.kind != VEXQ_E_COLUMN || c.column < 0 || c.column >= (int)t.cols.size()) return true;
        const vexq_zone_map& z = t.cols[c.column].zones[rg];
        if (!z.has_min_max) return true;
        int64_t lo, hi;
        int lk;
        if (!literal_int64(p.zn_nodes[ch(1)], &lo, &lk) || !literal_int64(p.zn_nodes[ch(2)], &hi, &lk)) return true;
        if ((int64_t)z.max < lo || (int64_t)z.min > hi) return e.op == 1;
        return true;
    }
    if (e.kind == VEXQ_E_BINARY && e.op >= VEXQ_OP_EQ && e.op <= VEXQ_OP_GE) {
        const vexq_expr& L = p.zn_nodes[ch(0)];
        const vexq_expr& R = p.zn_nodes[ch(1)];
        const vexq_expr *cr, *lit;
        bool rev = false;
        if (L.kind == VEXQ_E_COLUMN) { cr = &L; lit = &R; }
        else if (R.kind == VEXQ_E_COLUMN) { cr = &R; lit = &L; rev = true; }
        else return true;
        if (cr->column < 0 || cr->column >= (int)t.cols.size()) return true;
        const vexq_zone_map& z = t.cols[cr->column].zones[rg];
        if (!z.has_min_max) return true;
        int64_t v;
        int lk;
        if (!literal_int64(*lit, &v, &lk)) return true;
        if (t.cols[cr->column].type == VEXQ_TYPE_FLOAT64 && lk == VEXQ_LIT_INT) {
            double f = (double)v;
            std::memcpy(&v, &f, 8);
        }
        int64_t mn = (int64_t)z.min, mx = (int64_t)z.max;
        int op = e.op;
        if (rev) {
            if (op == VEXQ_OP_LT) op = VEXQ_OP_GT;
            else if (op == VEXQ_OP_LE) op = VEXQ_OP_GE;
            else if (op == VEXQ_OP_GT) op = VEXQ_OP_LT;
            else if (op == VEXQ_OP_GE) op = VEXQ_OP_LE;
        }
        switch (op) {
            case VEXQ_OP_EQ: return mn <= v && v <= mx;
            case VEXQ_OP_LT: return mn < v;
            case VEXQ_OP_LE: return mn <= v;
            case VEXQ_OP_GT: return mx > v;
            case VEXQ_OP_GE: return mx >= v;
            default: return true;
        }
    }
    return true;
}

bool zone_eval(const Plan& p, int root, const Table& t, int rg) { return root < 0 ? true : zone_rec(p, root, t, rg); }

void check_ranges(const Plan& p) {
    if ((p.t && p.t->range_epoch != p.range_epoch) || (p.bt && p.bt->range_epoch != p.brange_epoch))
        fail(VEXQ_EINVAL, "table values were re-filled outside the value ranges this plan was compiled for; compile the plan again");
}

void set_plan_constants(const Plan& p, VQParams& P) {
    {
        std::lock_guard<std::mutex> lk(p.hot_mu);
        for (int h = 0; h < VQ_MAXHOT; h++) P.hot[h] = h < (int)p.hot_keys.size() ? p.hot_keys[h] : ~0ull;
    }
    for (size_t i = 0; i < p.lits.size() && i < VQ_MAXLITS; i++) P.lit[i] = p.lits[i];
    for (size_t f = 0; f < p.fx_lsb.size() && f < 16; f++) P.fx_lsb[f] = p.fx_lsb[f];
    P.cache_n = p.smem_groups;
}

ScanSegs make_segments(const Table& t, const std::vector<uint8_t>& mask, int rg_start, int rg_end, int unit) {
    ScanSegs s;
    s.nchunks = walk_segments(t, [&](int rg) { return mask[rg] != 0; }, rg_start, rg_end, unit,
                              [&](long long a, long long b, long long c0) {
                                  s.seg.push_back(a);
                                  s.seg.push_back(b);
                                  s.seg.push_back(c0);
                                  s.rows += b - a;
                              });
    return s;
}

}  // namespace vq
