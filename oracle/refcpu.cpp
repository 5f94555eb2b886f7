// refcpu.cpp — TEST INFRASTRUCTURE ONLY: CPU oracle and timed CPU baseline.
//
// A restatement, in C++, of vexq's Go execution path for
//   TableScan → Filter → Project → HashAggregate            (planner.Physical)
//   ParallelHashAggregate (morsel-driven, partial + merge)  (exec/parallel.go)
//   HashJoin / ParallelHashJoinAggregate                    (exec/join*.go)
// Each function names the reference file:line it follows. The code is the
// checker for the GPU library and the timed CPU baseline in bench.py; the
// product never links it. Compile with -O3 -ffp-contract=off so every float
// operation rounds once, exactly as Go's separate BinOp evaluations do.

#include "refcpu.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <unordered_map>
#include <unordered_set>
#include <vector>

namespace {

thread_local std::string g_err;

struct Error : std::runtime_error {
    using std::runtime_error::runtime_error;
};

constexpr int kBlockRows = 1024;  // storage/format.go:8

// ---- dictionaries (storage/codec.go:45-246) ---------------------------------
struct Dict {
    std::vector<std::string> keys;
    std::unordered_map<std::string, uint32_t> index;
    uint32_t add(const std::string& s) {  // DictBuilder.Add, codec.go:57-65
        auto it = index.find(s);
        if (it != index.end()) return it->second;
        uint32_t c = (uint32_t)keys.size();
        index.emplace(s, c);
        keys.push_back(s);
        return c;
    }
    bool lookup(const std::string& s, uint32_t* c) const {
        auto it = index.find(s);
        if (it == index.end()) return false;
        *c = it->second;
        return true;
    }
};

// ---- vectors (exec/batch.go:115-189) ----------------------------------------
// One typed column vector of n physical rows; validity is one byte per row
// (the reference packs it into an LSB-first bitmap; the values are the same).
struct Vec {
    int type = 0;
    int n = 0;
    std::vector<int64_t> i64;
    std::vector<double> f64;
    std::vector<int32_t> i32;
    std::vector<uint32_t> codes;
    std::vector<uint8_t> bits;   // BoolVector values
    std::vector<uint8_t> valid;  // 1 = valid
    const Dict* dict = nullptr;
    std::shared_ptr<Dict> owned;
    void resize(int t, int rows) {
        type = t;
        n = rows;
        valid.assign(rows, 0);
        switch (t) {
            case VEXQ_TYPE_INT64: i64.assign(rows, 0); break;
            case VEXQ_TYPE_FLOAT64: f64.assign(rows, 0.0); break;
            case VEXQ_TYPE_DATE: i32.assign(rows, 0); break;
            case VEXQ_TYPE_STRING: codes.assign(rows, 0); break;
            case VEXQ_TYPE_BOOL: bits.assign(rows, 0); break;
        }
    }
    bool isNull(int i) const { return !valid[i]; }
    std::string str(int i) const { return dict ? dict->keys[codes[i]] : std::string(); }
};

// extractInt64 (exec/aggregate.go:1083-1099): raw int64 bits of a value.
int64_t extractInt64(const Vec& v, int i) {
    switch (v.type) {
        case VEXQ_TYPE_INT64: return v.i64[i];
        case VEXQ_TYPE_FLOAT64: { int64_t b; std::memcpy(&b, &v.f64[i], 8); return b; }
        case VEXQ_TYPE_DATE: return (int64_t)v.i32[i];
        case VEXQ_TYPE_BOOL: return v.bits[i] ? 1 : 0;
        default: return 0;
    }
}
inline double bitsToF(int64_t b) { double d; std::memcpy(&d, &b, 8); return d; }
inline int64_t fToBits(double d) { int64_t b; std::memcpy(&b, &d, 8); return b; }

struct Batch {
    std::vector<const Vec*> cols;
    int length = 0;     // logical rows
    int phys = 0;       // physical rows
    bool has_sel = false;
    std::vector<uint16_t> sel;
    int rg = -1;
    int rowAt(int i) const { return has_sel ? sel[i] : i; }
    int rows() const { return has_sel ? (int)sel.size() : length; }
};

// ---- tables ------------------------------------------------------------------
struct Column {
    std::string name;
    int type = 0;
    std::vector<int64_t> i64;
    std::vector<double> f64;
    std::vector<int32_t> i32;
    std::vector<uint32_t> codes;  // per-RG local dictionary codes
    std::vector<uint8_t> b8;
    std::vector<uint8_t> valid;   // per row
    bool nullable = false;
    std::vector<std::shared_ptr<Dict>> dicts;  // per RG (one shared dict in global mode)
    std::vector<vexq_zone_map> zones;          // per RG
};

struct Table {
    std::vector<Column> cols;
    int64_t nrows = 0;
    int rg_rows = 65536;
    int n_rg = 0;
    int64_t rgStart(int rg) const { return (int64_t)rg * rg_rows; }
    int64_t rgEnd(int rg) const { return std::min<int64_t>(nrows, (int64_t)(rg + 1) * rg_rows); }
};

// Zone maps with the writer's rules (storage/writer.go:205-372).
void computeZones(Table& t) {
    for (auto& c : t.cols) {
        c.zones.assign(t.n_rg, vexq_zone_map{});
        for (int rg = 0; rg < t.n_rg; rg++) {
            vexq_zone_map z{};
            int64_t s = t.rgStart(rg), e = t.rgEnd(rg);
            if (c.type == VEXQ_TYPE_INT64) {  // writeInt64Blocks :205-250
                for (int64_t r = s; r < e; r++) {
                    if (!c.valid[r]) { z.null_count++; continue; }
                    int64_t v = c.i64[r];
                    z.sum = (int64_t)((uint64_t)z.sum + (uint64_t)v);
                    if (!z.has_min_max) { z.min = z.max = (uint64_t)v; z.has_min_max = 1; }
                    else { if (v < (int64_t)z.min) z.min = (uint64_t)v; if (v > (int64_t)z.max) z.max = (uint64_t)v; }
                }
            } else if (c.type == VEXQ_TYPE_FLOAT64) {  // writeFloat64Blocks :252-300
                double sumF = 0, mn = 0, mx = 0;
                for (int64_t r = s; r < e; r++) {
                    if (!c.valid[r]) { z.null_count++; continue; }
                    double v = c.f64[r];
                    sumF += v;
                    if (!z.has_min_max) { mn = mx = v; z.has_min_max = 1; }
                    else { if (v < mn) mn = v; if (v > mx) mx = v; }
                }
                z.sum = fToBits(sumF);
                if (z.has_min_max) { z.min = (uint64_t)fToBits(mn); z.max = (uint64_t)fToBits(mx); }
            } else if (c.type == VEXQ_TYPE_DATE) {  // writeDateBlocks :302-338 (zero-extended)
                for (int64_t r = s; r < e; r++) {
                    if (!c.valid[r]) { z.null_count++; continue; }
                    int32_t v = c.i32[r];
                    uint64_t uv = (uint64_t)(uint32_t)v;
                    if (!z.has_min_max) { z.min = z.max = uv; z.has_min_max = 1; }
                    else { if ((int32_t)z.min > v) z.min = uv; if ((int32_t)z.max < v) z.max = uv; }
                }
            } else if (c.type == VEXQ_TYPE_STRING) {  // writeStringBlocks :363-378
                for (int64_t r = s; r < e; r++) if (!c.valid[r]) z.null_count++;
                size_t dl = c.dicts[rg]->keys.size();
                if (dl > 0) { z.has_min_max = 1; z.min = 0; z.max = dl - 1; }
            } else {  // bool: null count only
                for (int64_t r = s; r < e; r++) if (!c.valid[r]) z.null_count++;
            }
            c.zones[rg] = z;
        }
    }
}

// ---- plan descriptor access ----------------------------------------------------
struct Nodes {
    const vexq_expr* nodes;
    int nnodes;
    const int32_t* children;
    int nchildren;
    const vexq_expr& at(int i) const {
        if (i < 0 || i >= nnodes) throw Error("expression node index out of range");
        return nodes[i];
    }
    int child(const vexq_expr& n, int k) const {
        int idx = n.child0 + k;
        if (k >= n.nchildren || idx < 0 || idx >= nchildren) throw Error("expression child out of range");
        return children[idx];
    }
};

// Column references of an expression tree (pruneColumns, planner/optimizer.go).
void collectCols(const Nodes& N, int idx, std::vector<char>& need, int offset = 0, int limit = 1 << 30) {
    if (idx < 0) return;
    const vexq_expr& n = N.at(idx);
    if (n.kind == VEXQ_E_COLUMN) {
        int c = n.column - offset;
        if (c >= 0 && c < (int)need.size() && n.column < limit) need[c] = 1;
        return;
    }
    for (int k = 0; k < n.nchildren; k++) collectCols(N, N.child(n, k), need, offset, limit);
}

// time.ParseInLocation("2006-01-02", s, UTC) → days since epoch, strict.
bool parseDate(const char* s, int64_t* days) {
    if (!s || std::strlen(s) != 10 || s[4] != '-' || s[7] != '-') return false;
    for (int i : {0, 1, 2, 3, 5, 6, 8, 9}) if (s[i] < '0' || s[i] > '9') return false;
    int y = (s[0] - '0') * 1000 + (s[1] - '0') * 100 + (s[2] - '0') * 10 + (s[3] - '0');
    int m = (s[5] - '0') * 10 + (s[6] - '0');
    int d = (s[8] - '0') * 10 + (s[9] - '0');
    if (m < 1 || m > 12) return false;
    static const int md[12] = {31, 28, 31, 30, 31, 30, 31, 31, 30, 31, 30, 31};
    bool leap = (y % 4 == 0 && y % 100 != 0) || y % 400 == 0;
    int dim = md[m - 1] + ((m == 2 && leap) ? 1 : 0);
    if (d < 1 || d > dim) return false;
    // days from civil (proleptic Gregorian)
    int yy = y - (m <= 2);
    int era = (yy >= 0 ? yy : yy - 399) / 400;
    int yoe = yy - era * 400;
    int doy = (153 * (m + (m > 2 ? -3 : 9)) + 2) / 5 + d - 1;
    int doe = yoe * 365 + yoe / 4 - yoe / 100 + doy;
    *days = (int64_t)era * 146097 + doe - 719468;
    return true;
}

// ---- executable expressions (exec/expr.go) -------------------------------------
enum XK { XCOL, XLIT, XCMP, XARITH, XCAST, XAND, XOR, XNOT, XISNULL, XISNOTNULL, XIN, XLIKE, XSTREQ, XCASE };

struct X {
    XK k;
    int type = 0;  // result type
    int op = 0;
    int col = -1;
    int64_t li = 0;
    double lf = 0;
    int32_t ld = 0;
    bool lb = false;
    std::string ls;
    std::vector<std::unique_ptr<X>> ch;
    bool has_else = false;
    bool negate = false;
    int set_kind = 0;  // IN: 1 int, 2 float, 3 string
    std::vector<int64_t> set_i;
    std::vector<double> set_f;
    std::vector<std::string> set_s;
    Vec out;
    Dict litDict;
    bool isLiteral() const { return k == XLIT; }
};

using XP = std::unique_ptr<X>;

struct Schema {
    std::vector<int> types;
};

XP mkLit(int type) { XP x(new X); x->k = XLIT; x->type = type; return x; }

// coerceOneSide (planner/physical.go:782-818): coerce literal b to a's type.
void coerceOneSide(const X& a, XP& b) {
    if (b->k != XLIT) return;
    switch (a.type) {
        case VEXQ_TYPE_DATE:
            if (b->type == VEXQ_TYPE_STRING) {
                int64_t days;
                if (parseDate(b->ls.c_str(), &days)) {
                    XP n = mkLit(VEXQ_TYPE_DATE);
                    n->ld = (int32_t)days;
                    b = std::move(n);
                }
            } else if (b->type == VEXQ_TYPE_INT64) {
                XP n = mkLit(VEXQ_TYPE_DATE);
                n->ld = (int32_t)b->li;
                b = std::move(n);
            }
            break;
        case VEXQ_TYPE_FLOAT64:
            if (b->type == VEXQ_TYPE_INT64) {
                XP n = mkLit(VEXQ_TYPE_FLOAT64);
                n->lf = (double)b->li;
                b = std::move(n);
            }
            break;
        case VEXQ_TYPE_INT64:
            if (b->type == VEXQ_TYPE_FLOAT64) {
                XP n = mkLit(VEXQ_TYPE_INT64);
                double f = b->lf;
                // Go int64(f): truncation toward zero
                n->li = (std::isnan(f) || f >= 9.2233720368547758e18 || f < -9.2233720368547758e18)
                            ? std::numeric_limits<int64_t>::min()
                            : (int64_t)f;
                b = std::move(n);
            }
            break;
    }
}

bool isCmp(int op) { return op >= VEXQ_OP_EQ && op <= VEXQ_OP_GE; }

// buildExecExpr (planner/physical.go:376-547) and buildBinExpr (:549-620).
XP build(const Nodes& N, int idx, const Schema& s) {
    const vexq_expr& n = N.at(idx);
    switch (n.kind) {
        case VEXQ_E_COLUMN: {
            if (n.column < 0 || n.column >= (int)s.types.size()) throw Error("column index out of range");
            XP x(new X);
            x->k = XCOL;
            x->col = n.column;
            x->type = s.types[n.column];
            return x;
        }
        case VEXQ_E_LITERAL: {
            XP x(new X);
            x->k = XLIT;
            switch (n.lit_kind) {
                case VEXQ_LIT_INT: x->type = VEXQ_TYPE_INT64; x->li = n.lit_int; break;
                case VEXQ_LIT_FLOAT: x->type = VEXQ_TYPE_FLOAT64; x->lf = n.lit_float; break;
                case VEXQ_LIT_STRING: x->type = VEXQ_TYPE_STRING; x->ls = n.lit_str ? n.lit_str : ""; break;
                case VEXQ_LIT_BOOL: x->type = VEXQ_TYPE_BOOL; x->lb = n.lit_int != 0; break;
                default: throw Error("bad literal kind");
            }
            return x;
        }
        case VEXQ_E_AND:
        case VEXQ_E_OR: {
            XP x(new X);
            x->k = n.kind == VEXQ_E_AND ? XAND : XOR;
            x->type = VEXQ_TYPE_BOOL;
            for (int k = 0; k < n.nchildren; k++) {
                XP c = build(N, N.child(n, k), s);
                if (c->type != VEXQ_TYPE_BOOL) throw Error("AND/OR operand is not boolean");
                x->ch.push_back(std::move(c));
            }
            return x;
        }
        case VEXQ_E_NOT: {
            XP c = build(N, N.child(n, 0), s);
            if (c->type != VEXQ_TYPE_BOOL) throw Error("NOT requires a boolean operand");
            XP x(new X);
            x->k = XNOT;
            x->type = VEXQ_TYPE_BOOL;
            x->ch.push_back(std::move(c));
            return x;
        }
        case VEXQ_E_NEG: {  // unary minus → child * -1 (physical.go:414-436)
            XP c = build(N, N.child(n, 0), s);
            XP lit;
            if (c->type == VEXQ_TYPE_FLOAT64) { lit = mkLit(VEXQ_TYPE_FLOAT64); lit->lf = -1.0; }
            else if (c->type == VEXQ_TYPE_INT64) { lit = mkLit(VEXQ_TYPE_INT64); lit->li = -1; }
            else throw Error("unary minus not supported for type");
            XP x(new X);
            x->k = XARITH;
            x->op = VEXQ_OP_MUL;
            x->type = c->type;
            x->ch.push_back(std::move(c));
            x->ch.push_back(std::move(lit));
            return x;
        }
        case VEXQ_E_IS_NULL:
        case VEXQ_E_IS_NOT_NULL: {
            XP x(new X);
            x->k = n.kind == VEXQ_E_IS_NULL ? XISNULL : XISNOTNULL;
            x->type = VEXQ_TYPE_BOOL;
            x->ch.push_back(build(N, N.child(n, 0), s));
            return x;
        }
        case VEXQ_E_BETWEEN: {  // physical.go:446-469 + BetweenExpr (expr.go:1319-1339)
            XP c = build(N, N.child(n, 0), s);
            XP lo = build(N, N.child(n, 1), s);
            XP hi = build(N, N.child(n, 2), s);
            coerceOneSide(*c, lo);
            coerceOneSide(*c, hi);
            auto cmpNode = [](int op, const X& child, XP other) {
                XP b(new X);
                b->k = XCMP;
                b->op = op;
                b->type = VEXQ_TYPE_BOOL;
                b->ch.push_back(nullptr);  // placeholder for a shared child
                b->ch.push_back(std::move(other));
                (void)child;
                return b;
            };
            // The rewritten AND shares the child expression; build it twice
            // from the descriptor (column refs and pure expressions evaluate
            // identically).
            XP c2 = build(N, N.child(n, 0), s);
            XP ge = cmpNode(VEXQ_OP_GE, *c, std::move(lo));
            ge->ch[0] = std::move(c);
            XP le = cmpNode(VEXQ_OP_LE, *c2, std::move(hi));
            le->ch[0] = std::move(c2);
            for (auto* b : {ge.get(), le.get()}) {
                int lt = b->ch[0]->type, rt = b->ch[1]->type;
                if (lt != rt || lt == VEXQ_TYPE_STRING || lt == VEXQ_TYPE_BOOL)
                    throw Error("BETWEEN operand types not comparable");
            }
            XP a(new X);
            a->k = XAND;
            a->type = VEXQ_TYPE_BOOL;
            a->ch.push_back(std::move(ge));
            a->ch.push_back(std::move(le));
            if (n.op == 1) {
                XP x(new X);
                x->k = XNOT;
                x->type = VEXQ_TYPE_BOOL;
                x->ch.push_back(std::move(a));
                return x;
            }
            return a;
        }
        case VEXQ_E_IN: {  // physical.go:470-491 + InExpr (expr.go:1191-1243)
            XP c = build(N, N.child(n, 0), s);
            XP x(new X);
            x->k = XIN;
            x->type = VEXQ_TYPE_BOOL;
            int kind = 0;
            for (int k = 1; k < n.nchildren; k++) {
                const vexq_expr& l = N.at(N.child(n, k));
                if (l.kind != VEXQ_E_LITERAL) continue;  // non-literals are skipped by the planner
                int lk = l.lit_kind == VEXQ_LIT_INT ? 1 : l.lit_kind == VEXQ_LIT_FLOAT ? 2
                         : l.lit_kind == VEXQ_LIT_STRING ? 3 : 0;
                if (!lk) continue;
                if (kind && kind != lk) throw Error("IN list mixes literal types");
                kind = lk;
                if (lk == 1) x->set_i.push_back(l.lit_int);
                if (lk == 2) x->set_f.push_back(l.lit_float);
                if (lk == 3) x->set_s.push_back(l.lit_str ? l.lit_str : "");
            }
            // A mismatch between the column and literal types is a type
            // assertion panic in the reference; reject it.
            if (kind && ((c->type == VEXQ_TYPE_INT64 && kind != 1) || (c->type == VEXQ_TYPE_FLOAT64 && kind != 2) ||
                         (c->type == VEXQ_TYPE_STRING && kind != 3)))
                throw Error("IN literal type does not match the operand");
            x->set_kind = kind;
            x->ch.push_back(std::move(c));
            if (n.op == 1) {
                XP y(new X);
                y->k = XNOT;
                y->type = VEXQ_TYPE_BOOL;
                y->ch.push_back(std::move(x));
                return y;
            }
            return x;
        }
        case VEXQ_E_LIKE: {
            XP c = build(N, N.child(n, 0), s);
            const vexq_expr& p = N.at(N.child(n, 1));
            if (p.kind != VEXQ_E_LITERAL || p.lit_kind != VEXQ_LIT_STRING) throw Error("LIKE pattern must be a string literal");
            if (c->type != VEXQ_TYPE_STRING) throw Error("LIKE requires STRING column");
            XP x(new X);
            x->k = XLIKE;
            x->type = VEXQ_TYPE_BOOL;
            x->ls = p.lit_str ? p.lit_str : "";
            x->ch.push_back(std::move(c));
            if (n.op == 1) {
                XP y(new X);
                y->k = XNOT;
                y->type = VEXQ_TYPE_BOOL;
                y->ch.push_back(std::move(x));
                return y;
            }
            return x;
        }
        case VEXQ_E_CASE: {  // physical.go:508-546
            XP x(new X);
            x->k = XCASE;
            x->has_else = n.op == 1;
            int nw = (n.nchildren - (x->has_else ? 1 : 0)) / 2;
            for (int w = 0; w < nw; w++) {
                XP cond = build(N, N.child(n, 2 * w), s);
                XP res = build(N, N.child(n, 2 * w + 1), s);
                x->ch.push_back(std::move(cond));
                x->ch.push_back(std::move(res));
            }
            if (x->has_else) x->ch.push_back(build(N, N.child(n, n.nchildren - 1), s));
            int t = nw > 0 ? x->ch[1]->type : VEXQ_TYPE_FLOAT64;
            for (int w = 0; w < nw; w++)
                if (x->ch[2 * w + 1]->type != t) throw Error("CASE branches must have a common type");
            if (x->has_else && x->ch.back()->type != t) throw Error("CASE ELSE type mismatch");
            if (t != VEXQ_TYPE_INT64 && t != VEXQ_TYPE_FLOAT64 && t != VEXQ_TYPE_STRING)
                throw Error("CASE result type not supported");
            x->type = t;
            return x;
        }
        case VEXQ_E_BINARY: {
            XP l = build(N, N.child(n, 0), s);
            XP r = build(N, N.child(n, 1), s);
            // coercePair (physical.go:773-778)
            coerceOneSide(*l, r);
            coerceOneSide(*r, l);
            if ((n.op == VEXQ_OP_EQ || n.op == VEXQ_OP_NE) && l->type == VEXQ_TYPE_STRING && r->type == VEXQ_TYPE_STRING) {
                X* col = nullptr;
                X* lit = nullptr;
                if (l->k == XCOL && r->k == XLIT) { col = l.get(); lit = r.get(); }
                else if (r->k == XCOL && l->k == XLIT) { col = r.get(); lit = l.get(); }
                if (col) {  // StringEqExpr (expr.go:1342-1388)
                    XP x(new X);
                    x->k = XSTREQ;
                    x->type = VEXQ_TYPE_BOOL;
                    x->col = col->col;
                    x->ls = lit->ls;
                    x->negate = n.op == VEXQ_OP_NE;
                    return x;
                }
                throw Error("cmp not supported for string operands");
            }
            if (n.op < VEXQ_OP_EQ || n.op > VEXQ_OP_DIV) throw Error("unknown binary op");
            XP x(new X);
            x->op = n.op;
            if (isCmp(n.op)) {
                x->k = XCMP;
                x->type = VEXQ_TYPE_BOOL;
                int lt = l->type, rt = r->type;
                if (lt != rt || lt == VEXQ_TYPE_STRING || lt == VEXQ_TYPE_BOOL)
                    throw Error("comparison operand types not comparable");
            } else {
                x->k = XARITH;
                int rt = l->type;
                if (l->type == VEXQ_TYPE_FLOAT64 || r->type == VEXQ_TYPE_FLOAT64) rt = VEXQ_TYPE_FLOAT64;
                if (rt == VEXQ_TYPE_FLOAT64) {
                    auto cast = [](XP& e) {
                        if (e->type == VEXQ_TYPE_INT64) {
                            XP c(new X);
                            c->k = XCAST;
                            c->type = VEXQ_TYPE_FLOAT64;
                            c->ch.push_back(std::move(e));
                            e = std::move(c);
                        }
                    };
                    cast(l);
                    cast(r);
                }
                if (l->type != r->type || (l->type != VEXQ_TYPE_INT64 && l->type != VEXQ_TYPE_FLOAT64))
                    throw Error("arithmetic operand types not supported");
                x->type = rt;
            }
            x->ch.push_back(std::move(l));
            x->ch.push_back(std::move(r));
            return x;
        }
    }
    throw Error("unsupported expression kind");
}

// likeMatch (expr.go:1277-1311)
bool likeMatch(const char* p, size_t pn, const char* s, size_t sn) {
    while (pn > 0) {
        if (p[0] == '%') {
            p++; pn--;
            if (pn == 0) return true;
            for (size_t i = 0; i <= sn; i++)
                if (likeMatch(p, pn, s + i, sn - i)) return true;
            return false;
        } else if (p[0] == '_') {
            if (sn == 0) return false;
            p++; pn--; s++; sn--;
        } else {
            if (sn == 0 || p[0] != s[0]) return false;
            p++; pn--; s++; sn--;
        }
    }
    return sn == 0;
}

template <class T>
bool cmpOp(int op, T a, T b) {
    switch (op) {
        case VEXQ_OP_EQ: return a == b;
        case VEXQ_OP_NE: return a != b;
        case VEXQ_OP_LT: return a < b;
        case VEXQ_OP_LE: return a <= b;
        case VEXQ_OP_GT: return a > b;
        case VEXQ_OP_GE: return a >= b;
    }
    return false;
}

// Eval (exec/expr.go): evaluates over the batch's PHYSICAL rows.
const Vec* eval(X* x, const Batch& b) {
    const int n = b.phys;
    Vec& o = x->out;
    switch (x->k) {
        case XCOL:
            return b.cols[x->col];
        case XLIT: {  // Literal.Eval (expr.go:86-185)
            if (o.n != n || o.type != x->type) {
                o.resize(x->type, n);
                std::fill(o.valid.begin(), o.valid.end(), 1);
                switch (x->type) {
                    case VEXQ_TYPE_INT64: std::fill(o.i64.begin(), o.i64.end(), x->li); break;
                    case VEXQ_TYPE_FLOAT64: std::fill(o.f64.begin(), o.f64.end(), x->lf); break;
                    case VEXQ_TYPE_DATE: std::fill(o.i32.begin(), o.i32.end(), x->ld); break;
                    case VEXQ_TYPE_BOOL: std::fill(o.bits.begin(), o.bits.end(), x->lb ? 1 : 0); break;
                    case VEXQ_TYPE_STRING:
                        if (x->litDict.keys.empty()) x->litDict.add(x->ls);
                        o.dict = &x->litDict;
                        break;
                }
            }
            return &o;
        }
        case XCAST: {  // CastIntToFloatExpr (expr.go:194-219)
            const Vec* v = eval(x->ch[0].get(), b);
            o.resize(VEXQ_TYPE_FLOAT64, v->n);
            for (int i = 0; i < v->n; i++) { o.f64[i] = (double)v->i64[i]; o.valid[i] = v->valid[i]; }
            return &o;
        }
        case XCMP: {  // evalCmp (expr.go:287-318): bit = cmp & valid
            const Vec* l = eval(x->ch[0].get(), b);
            const Vec* r = eval(x->ch[1].get(), b);
            int m = l->n;
            o.resize(VEXQ_TYPE_BOOL, m);
            for (int i = 0; i < m; i++) {
                uint8_t v = l->valid[i] & r->valid[i];
                o.valid[i] = v;
                if (!v) continue;
                bool c;
                switch (l->type) {
                    case VEXQ_TYPE_INT64: c = cmpOp(x->op, l->i64[i], r->i64[i]); break;
                    case VEXQ_TYPE_FLOAT64: c = cmpOp(x->op, l->f64[i], r->f64[i]); break;
                    default: c = cmpOp(x->op, l->i32[i], r->i32[i]); break;
                }
                o.bits[i] = c ? 1 : 0;
            }
            return &o;
        }
        case XARITH: {  // evalArith / applyArith* (expr.go:956-1026)
            const Vec* l = eval(x->ch[0].get(), b);
            const Vec* r = eval(x->ch[1].get(), b);
            int m = l->n;
            o.resize(x->type, m);
            for (int i = 0; i < m; i++) {
                uint8_t v = l->valid[i] & r->valid[i];
                o.valid[i] = v;
                if (!v) continue;
                if (x->type == VEXQ_TYPE_INT64) {
                    uint64_t a = (uint64_t)l->i64[i], c = (uint64_t)r->i64[i];
                    int64_t res = 0;
                    switch (x->op) {
                        case VEXQ_OP_ADD: res = (int64_t)(a + c); break;
                        case VEXQ_OP_SUB: res = (int64_t)(a - c); break;
                        case VEXQ_OP_MUL: res = (int64_t)(a * c); break;
                        case VEXQ_OP_DIV: {
                            int64_t aa = l->i64[i], cc = r->i64[i];
                            if (cc == 0) res = 0;
                            else if (cc == -1) res = (int64_t)(0 - a);  // Go: MinInt64/-1 wraps
                            else res = aa / cc;
                            break;
                        }
                    }
                    o.i64[i] = res;
                } else {
                    double a = l->f64[i], c = r->f64[i], res = 0;
                    switch (x->op) {
                        case VEXQ_OP_ADD: res = a + c; break;
                        case VEXQ_OP_SUB: res = a - c; break;
                        case VEXQ_OP_MUL: res = a * c; break;
                        case VEXQ_OP_DIV: res = (c == 0) ? std::numeric_limits<double>::quiet_NaN() : a / c; break;
                    }
                    o.f64[i] = res;
                }
            }
            return &o;
        }
        case XAND:
        case XOR: {  // AndExpr / OrExpr (expr.go:1030-1108)
            const Vec* f = eval(x->ch[0].get(), b);
            int m = f->n;
            o.resize(VEXQ_TYPE_BOOL, m);
            for (int i = 0; i < m; i++) { o.bits[i] = f->bits[i]; o.valid[i] = f->valid[i]; }
            for (size_t k = 1; k < x->ch.size(); k++) {
                const Vec* c = eval(x->ch[k].get(), b);
                if (x->k == XAND)
                    for (int i = 0; i < m; i++) { o.bits[i] &= c->bits[i]; o.valid[i] &= c->valid[i]; }
                else
                    for (int i = 0; i < m; i++) { o.bits[i] |= c->bits[i]; o.valid[i] |= c->valid[i]; }
            }
            return &o;
        }
        case XNOT: {  // NotExpr (expr.go:1117-1140): flip only valid bits
            const Vec* c = eval(x->ch[0].get(), b);
            o.resize(VEXQ_TYPE_BOOL, c->n);
            for (int i = 0; i < c->n; i++) { o.valid[i] = c->valid[i]; o.bits[i] = c->bits[i] ^ c->valid[i]; }
            return &o;
        }
        case XISNULL:
        case XISNOTNULL: {
            const Vec* c = eval(x->ch[0].get(), b);
            o.resize(VEXQ_TYPE_BOOL, c->n);
            for (int i = 0; i < c->n; i++) {
                o.valid[i] = 1;
                bool isn = c->isNull(i);
                o.bits[i] = (x->k == XISNULL) ? isn : !isn;
            }
            return &o;
        }
        case XIN: {  // InExpr (expr.go:1204-1243)
            const Vec* c = eval(x->ch[0].get(), b);
            o.resize(VEXQ_TYPE_BOOL, c->n);
            for (int i = 0; i < c->n; i++) {
                if (c->isNull(i)) continue;
                o.valid[i] = 1;
                bool found = false;
                if (c->type == VEXQ_TYPE_INT64) {
                    for (auto v : x->set_i) if (c->i64[i] == v) { found = true; break; }
                } else if (c->type == VEXQ_TYPE_FLOAT64) {
                    for (auto v : x->set_f) if (c->f64[i] == v) { found = true; break; }
                } else if (c->type == VEXQ_TYPE_STRING) {
                    const std::string& sv = c->dict ? c->dict->keys[c->codes[i]] : std::string();
                    for (auto& v : x->set_s) if (sv == v) { found = true; break; }
                }
                o.bits[i] = found;
            }
            return &o;
        }
        case XLIKE: {
            const Vec* c = eval(x->ch[0].get(), b);
            o.resize(VEXQ_TYPE_BOOL, c->n);
            for (int i = 0; i < c->n; i++) {
                if (c->isNull(i)) continue;
                o.valid[i] = 1;
                std::string s = c->str(i);
                o.bits[i] = likeMatch(x->ls.data(), x->ls.size(), s.data(), s.size());
            }
            return &o;
        }
        case XSTREQ: {  // StringEqExpr (expr.go:1356-1388): per-dictionary lookup
            const Vec* c = b.cols[x->col];
            o.resize(VEXQ_TYPE_BOOL, c->n);
            if (!c->dict) return &o;
            uint32_t code;
            if (!c->dict->lookup(x->ls, &code)) {
                if (x->negate)
                    for (int i = 0; i < c->n; i++) { o.valid[i] = 1; o.bits[i] = 1; }
                return &o;
            }
            for (int i = 0; i < c->n; i++) {
                if (c->isNull(i)) continue;
                o.valid[i] = 1;
                bool m = c->codes[i] == code;
                o.bits[i] = x->negate ? !m : m;
            }
            return &o;
        }
        case XCASE: {  // CaseExpr + mergeVectors (expr.go:1405-1503)
            int t = x->type;
            int nw = (int)(x->ch.size() - (x->has_else ? 1 : 0)) / 2;
            Vec cur;
            if (x->has_else) {
                const Vec* e = eval(x->ch.back().get(), b);
                cur = *e;
                cur.owned.reset();
            } else {
                cur.resize(t, n);  // nullVector: all NULL
            }
            for (int w = nw - 1; w >= 0; w--) {
                const Vec* cond = eval(x->ch[2 * w].get(), b);
                const Vec* val = eval(x->ch[2 * w + 1].get(), b);
                if (t == VEXQ_TYPE_STRING) {
                    auto db = std::make_shared<Dict>();
                    std::vector<uint32_t> baseRemap, valRemap;
                    if (cur.dict) for (auto& s : cur.dict->keys) baseRemap.push_back(db->add(s));
                    if (val->dict) for (auto& s : val->dict->keys) valRemap.push_back(db->add(s));
                    Vec nx;
                    nx.resize(t, n);
                    for (int i = 0; i < n; i++) {
                        if (cond->valid[i] && cond->bits[i]) {
                            if (!val->isNull(i)) { nx.codes[i] = valRemap[val->codes[i]]; nx.valid[i] = 1; }
                        } else if (!cur.isNull(i)) {
                            nx.codes[i] = baseRemap[cur.codes[i]];
                            nx.valid[i] = 1;
                        }
                    }
                    nx.owned = db;
                    nx.dict = db.get();
                    cur = std::move(nx);
                } else {
                    for (int i = 0; i < n; i++) {
                        if (cond->valid[i] && cond->bits[i]) {
                            if (t == VEXQ_TYPE_INT64) cur.i64[i] = val->i64[i];
                            else cur.f64[i] = val->f64[i];
                            cur.valid[i] = val->valid[i];
                        }
                    }
                }
            }
            o = std::move(cur);
            return &o;
        }
    }
    return &o;
}

// ---- zone predicate (planner/physical.go:624-750) -----------------------------------
bool literalInt64(const vexq_expr& e, int64_t* v, int* litKind) {
    if (e.kind != VEXQ_E_LITERAL) return false;
    *litKind = e.lit_kind;
    if (e.lit_kind == VEXQ_LIT_INT) { *v = e.lit_int; return true; }
    if (e.lit_kind == VEXQ_LIT_FLOAT) { *v = fToBits(e.lit_float); return true; }
    if (e.lit_kind == VEXQ_LIT_STRING) return parseDate(e.lit_str, v);
    return false;
}

bool zoneEval(const Nodes& N, int idx, const Table& t, int rg) {
    const vexq_expr& e = N.at(idx);
    if (e.kind == VEXQ_E_AND) {
        for (int k = 0; k < e.nchildren; k++) if (!zoneEval(N, N.child(e, k), t, rg)) return false;
        return true;
    }
    if (e.kind == VEXQ_E_OR) {
        if (e.nchildren == 0) return true;
        for (int k = 0; k < e.nchildren; k++) if (zoneEval(N, N.child(e, k), t, rg)) return true;
        return false;
    }
    if (e.kind == VEXQ_E_BETWEEN) {
        const vexq_expr& c = N.at(N.child(e, 0));
        if (c.kind != VEXQ_E_COLUMN || c.column < 0 || c.column >= (int)t.cols.size()) return true;
        const vexq_zone_map& zm = t.cols[c.column].zones[rg];
        if (!zm.has_min_max) return true;
        int64_t lo, hi;
        int lk;
        if (!literalInt64(N.at(N.child(e, 1)), &lo, &lk) || !literalInt64(N.at(N.child(e, 2)), &hi, &lk)) return true;
        if ((int64_t)zm.max < lo || (int64_t)zm.min > hi) return e.op == 1;
        return true;
    }
    if (e.kind == VEXQ_E_BINARY && isCmp(e.op)) {
        const vexq_expr& L = N.at(N.child(e, 0));
        const vexq_expr& R = N.at(N.child(e, 1));
        const vexq_expr* cr = nullptr;
        const vexq_expr* lit = nullptr;
        bool reversed = false;
        if (L.kind == VEXQ_E_COLUMN) { cr = &L; lit = &R; }
        else if (R.kind == VEXQ_E_COLUMN) { cr = &R; lit = &L; reversed = true; }
        else return true;
        if (cr->column < 0 || cr->column >= (int)t.cols.size()) return true;
        const vexq_zone_map& zm = t.cols[cr->column].zones[rg];
        if (!zm.has_min_max) return true;
        int64_t v;
        int lk;
        if (!literalInt64(*lit, &v, &lk)) return true;
        if (t.cols[cr->column].type == VEXQ_TYPE_FLOAT64 && lk == VEXQ_LIT_INT) v = fToBits((double)v);
        int64_t mn = (int64_t)zm.min, mx = (int64_t)zm.max;
        int op = e.op;
        if (reversed) {
            if (op == VEXQ_OP_LT) op = VEXQ_OP_GT;
            else if (op == VEXQ_OP_LE) op = VEXQ_OP_GE;
            else if (op == VEXQ_OP_GT) op = VEXQ_OP_LT;
            else if (op == VEXQ_OP_GE) op = VEXQ_OP_LE;
        }
        switch (op) {
            case VEXQ_OP_EQ: return mn <= v && v <= mx;
            case VEXQ_OP_NE: return true;
            case VEXQ_OP_LT: return mn < v;
            case VEXQ_OP_LE: return mn <= v;
            case VEXQ_OP_GT: return mx > v;
            case VEXQ_OP_GE: return mx >= v;
        }
        return true;
    }
    return true;
}

// ---- TableScan (exec/scan.go:199-409): 1024-row batches per row group ----------
struct Scan {
    const Table* t;
    std::vector<Vec> bufs;
    std::vector<const Vec*> ptrs;
    std::vector<char> need;  // projected columns (optimizer column pruning); empty = all
    explicit Scan(const Table* tt, std::vector<char> nd = {}) : t(tt), bufs(tt->cols.size()), need(std::move(nd)) {
        for (auto& v : bufs) ptrs.push_back(&v);
    }
    // Decodes rows [s, s+n) of row group rg into the reused buffers.
    void load(int rg, int64_t s, int n, Batch& b) {
        for (size_t c = 0; c < t->cols.size(); c++) {
            if (!need.empty() && !need[c]) continue;
            const Column& col = t->cols[c];
            Vec& v = bufs[c];
            v.type = col.type;
            v.n = n;
            v.valid.resize(n);
            std::memcpy(v.valid.data(), col.valid.data() + s, n);
            switch (col.type) {
                case VEXQ_TYPE_INT64: v.i64.resize(n); std::memcpy(v.i64.data(), col.i64.data() + s, n * 8); break;
                case VEXQ_TYPE_FLOAT64: v.f64.resize(n); std::memcpy(v.f64.data(), col.f64.data() + s, n * 8); break;
                case VEXQ_TYPE_DATE: v.i32.resize(n); std::memcpy(v.i32.data(), col.i32.data() + s, n * 4); break;
                case VEXQ_TYPE_STRING:
                    v.codes.resize(n);
                    std::memcpy(v.codes.data(), col.codes.data() + s, n * 4);
                    v.dict = col.dicts[rg].get();
                    break;
                case VEXQ_TYPE_BOOL: v.bits.resize(n); std::memcpy(v.bits.data(), col.b8.data() + s, n); break;
            }
        }
        b.cols = ptrs;
        b.length = n;
        b.phys = n;
        b.has_sel = false;
        b.sel.clear();
        b.rg = rg;
    }
};

// ---- aggregation (exec/aggregate.go, exec/agg_intkey.go) ------------------------
struct AggSpec {
    int kind;
    int accum;     // AccumTypeFor (aggregate.go:51-72)
    int srcType;   // input type (TypeInt64 for COUNT(*))
    int outType;   // schema type (aggregate.go:161-175)
    bool star;     // COUNT(*)
    std::string name;
};

int accumTypeFor(int kind, int src) {
    switch (kind) {
        case VEXQ_AGG_AVG: return VEXQ_TYPE_FLOAT64;
        case VEXQ_AGG_SUM: return src == VEXQ_TYPE_FLOAT64 ? VEXQ_TYPE_FLOAT64 : VEXQ_TYPE_INT64;
        case VEXQ_AGG_MIN:
        case VEXQ_AGG_MAX:
            if (src == VEXQ_TYPE_FLOAT64) return VEXQ_TYPE_FLOAT64;
            if (src == VEXQ_TYPE_STRING) return VEXQ_TYPE_STRING;
            return VEXQ_TYPE_INT64;
        default: return VEXQ_TYPE_INT64;
    }
}

struct GroupByVal {
    bool isNull = false;
    std::string str;
    uint64_t bits = 0;
};

// Shewchuk's exact summation (the algorithm behind Python's math.fsum).
struct ExactSum {
    std::vector<double> p;
    int special = 0;  // bit0: NaN, bit1: +inf, bit2: -inf
    void add(double x) {
        if (!std::isfinite(x)) {
            if (std::isnan(x)) special |= 1;
            else special |= x > 0 ? 2 : 4;
            return;
        }
        size_t i = 0;
        for (double y : p) {
            if (std::fabs(x) < std::fabs(y)) std::swap(x, y);
            double hi = x + y;
            double lo = y - (hi - x);
            if (lo != 0.0) p[i++] = lo;
            x = hi;
        }
        p.resize(i);
        p.push_back(x);
    }
    double value() const {
        if (special & 1 || (special & 6) == 6) return std::numeric_limits<double>::quiet_NaN();
        if (special & 2) return INFINITY;
        if (special & 4) return -INFINITY;
        if (p.empty()) return 0.0;
        // msum rounding: sum partials from the top with half-way correction
        int n = (int)p.size();
        double hi = p[n - 1], lo = 0;
        int i = n - 1;
        while (i > 0) {
            double x = hi, y = p[--i];
            hi = x + y;
            double yr = hi - x;
            lo = y - yr;
            if (lo != 0.0) break;
        }
        if (i > 0 && ((lo < 0 && p[i - 1] < 0) || (lo > 0 && p[i - 1] > 0))) {
            double y = lo * 2;
            double x = hi + y;
            double yr = x - hi;
            if (y == yr) hi = x;
        }
        return hi;
    }
};

struct Group {
    std::vector<int64_t> accs;
    std::vector<int64_t> nonNull;
    std::vector<GroupByVal> sample;
    std::vector<std::string> strs;
    std::vector<ExactSum> exact;  // serial only, per agg (SUM/AVG float)
    // COUNT(DISTINCT) sets (aggregate.go:117-124): raw int64 images, or the
    // resolved strings of STRING inputs
    std::vector<std::unordered_set<int64_t>> dints;
    std::vector<std::unordered_set<std::string>> dstrs;
};

struct HashAgg {
    std::vector<int> groupBy;
    std::vector<AggSpec> aggs;
    std::vector<int> gbTypes;
    bool hasStrAgg = false;
    bool trackExact = false;
    std::vector<std::string> keys;
    std::unordered_map<std::string, Group> groups;

    // integer-key state (agg_intkey.go:19-47)
    bool ikEnabled = false, ikDecided = false;
    std::vector<Dict> globalDicts;
    std::vector<uint8_t> shifts, widths;
    std::vector<std::map<const Dict*, std::vector<uint32_t>>> remaps;
    std::vector<uint64_t> intKeys;
    std::unordered_map<uint64_t, Group> intGroups;

    void initMaps() {  // aggregate.go:222-249
        keys.clear();
        groups.clear();
        ikDecided = false;
        ikEnabled = false;
        intKeys.clear();
        intGroups.clear();
        hasStrAgg = false;
        for (auto& a : aggs) if (a.accum == VEXQ_TYPE_STRING) hasStrAgg = true;
    }

    Group newGroup() const {  // newAccums (aggregate.go:255-279)
        Group g;
        g.accs.assign(aggs.size(), 0);
        g.nonNull.assign(aggs.size(), 0);
        for (size_t j = 0; j < aggs.size(); j++) {
            const AggSpec& a = aggs[j];
            if (a.kind == VEXQ_AGG_MIN) {
                if (a.accum == VEXQ_TYPE_FLOAT64) g.accs[j] = fToBits(std::numeric_limits<double>::max());
                else if (a.accum != VEXQ_TYPE_STRING) g.accs[j] = std::numeric_limits<int64_t>::max();
            } else if (a.kind == VEXQ_AGG_MAX) {
                if (a.accum == VEXQ_TYPE_FLOAT64) g.accs[j] = fToBits(-std::numeric_limits<double>::max());
                else if (a.accum != VEXQ_TYPE_STRING) g.accs[j] = std::numeric_limits<int64_t>::min();
            }
        }
        if (hasStrAgg) g.strs.assign(aggs.size(), std::string());
        if (trackExact) g.exact.assign(aggs.size(), ExactSum());
        if (hasDistinct()) {
            g.dints.resize(aggs.size());
            g.dstrs.resize(aggs.size());
        }
        return g;
    }

    bool hasDistinct() const {
        for (auto& a : aggs) if (a.kind == VEXQ_AGG_COUNT_DISTINCT) return true;
        return false;
    }

    // COUNT(DISTINCT) fold of one row (aggregate.go:474-493): NULLs are not
    // in the set; strings by their value, other types by extractInt64
    static void foldDistinct(Group& g, size_t j, const Vec* v, int r) {
        if (v->isNull(r)) return;
        if (v->type == VEXQ_TYPE_STRING) g.dstrs[j].insert(v->str(r));
        else g.dints[j].insert(extractInt64(*v, r));
    }

    static void minMaxString(std::vector<std::string>& strs, size_t j, const std::string& s, bool seen, bool less) {
        if (!seen) { strs[j] = s; return; }
        if (less) { if (s < strs[j]) strs[j] = s; }
        else if (s > strs[j]) strs[j] = s;
    }

    // foldRow (agg_intkey.go:303-361)
    void foldRow(Group& g, const std::vector<const Vec*>& av, int r) {
        for (size_t j = 0; j < aggs.size(); j++) {
            const AggSpec& a = aggs[j];
            const Vec* v = av[j];
            switch (a.kind) {
                case VEXQ_AGG_COUNT:
                    if (a.star || !v->isNull(r)) { g.accs[j]++; g.nonNull[j]++; }
                    break;
                case VEXQ_AGG_COUNT_DISTINCT:
                    foldDistinct(g, j, v, r);
                    break;
                case VEXQ_AGG_SUM:
                    if (v->isNull(r)) break;
                    g.nonNull[j]++;
                    if (a.accum == VEXQ_TYPE_FLOAT64) {
                        g.accs[j] = fToBits(bitsToF(g.accs[j]) + v->f64[r]);
                        if (trackExact) g.exact[j].add(v->f64[r]);
                    } else {
                        g.accs[j] = (int64_t)((uint64_t)g.accs[j] + (uint64_t)extractInt64(*v, r));
                    }
                    break;
                case VEXQ_AGG_AVG: {
                    if (v->isNull(r)) break;
                    g.nonNull[j]++;
                    double x = v->type == VEXQ_TYPE_FLOAT64 ? v->f64[r] : (double)extractInt64(*v, r);
                    g.accs[j] = fToBits(bitsToF(g.accs[j]) + x);
                    if (trackExact) g.exact[j].add(x);
                    break;
                }
                case VEXQ_AGG_MIN:
                case VEXQ_AGG_MAX: {
                    if (v->isNull(r)) break;
                    bool less = a.kind == VEXQ_AGG_MIN;
                    if (a.accum == VEXQ_TYPE_STRING) {
                        minMaxString(g.strs, j, v->str(r), g.nonNull[j] > 0, less);
                        g.nonNull[j]++;
                        break;
                    }
                    g.nonNull[j]++;
                    int64_t val = extractInt64(*v, r);
                    if (a.accum == VEXQ_TYPE_FLOAT64) {
                        double cur = bitsToF(g.accs[j]), fv = bitsToF(val);
                        if ((less && fv < cur) || (!less && fv > cur)) g.accs[j] = val;
                    } else if ((less && val < g.accs[j]) || (!less && val > g.accs[j])) {
                        g.accs[j] = val;
                    }
                    break;
                }
            }
        }
    }

    // buildKey (aggregate.go:753-778)
    std::string buildKey(const Batch& b, int r) const {
        std::string k;
        for (int c : groupBy) {
            const Vec* v = b.cols[c];
            if (v->isNull(r)) { k.push_back((char)0x00); k.push_back((char)0xFF); }
            else if (v->type == VEXQ_TYPE_STRING) {
                std::string s = v->str(r);
                k.push_back((char)0x02);
                uint32_t len = (uint32_t)s.size();
                k.append((const char*)&len, 4);
                k += s;
                k.push_back((char)0xFF);
            } else {
                k.push_back((char)0x01);
                uint64_t u = (uint64_t)extractInt64(*v, r);
                k.append((const char*)&u, 8);
                k.push_back((char)0xFF);
            }
        }
        return k;
    }

    std::vector<GroupByVal> sampleOf(const Batch& b, int r) const {
        std::vector<GroupByVal> s(groupBy.size());
        for (size_t si = 0; si < groupBy.size(); si++) {
            const Vec* v = b.cols[groupBy[si]];
            if (v->isNull(r)) s[si].isNull = true;
            else if (v->type == VEXQ_TYPE_STRING) s[si].str = v->str(r);
            else s[si].bits = (uint64_t)extractInt64(*v, r);
        }
        return s;
    }

    // accumulateOneRow (agg_intkey.go:380-410)
    void accumulateOneRow(const std::string& key, const Batch& b, int r, const std::vector<const Vec*>& av) {
        auto it = groups.find(key);
        if (it == groups.end()) {
            Group g = newGroup();
            g.sample = sampleOf(b, r);
            it = groups.emplace(key, std::move(g)).first;
            keys.push_back(key);
        }
        foldRow(it->second, av, r);
    }

    void initIntKey(int n) {  // intKeyState.init (agg_intkey.go:67-100)
        intKeys.clear();
        intGroups.clear();
        globalDicts.assign(n, Dict());
        shifts.assign(n, 0);
        widths.assign(n, 0);
        remaps.assign(n, {});
        if (n <= 2) for (int i = 0; i < n; i++) { shifts[i] = (uint8_t)(i * 32); widths[i] = 32; }
        else if (n <= 4) for (int i = 0; i < n; i++) { shifts[i] = (uint8_t)(i * 16); widths[i] = 16; }
        else for (int i = 0; i < n; i++) { shifts[i] = (uint8_t)(i * 8); widths[i] = 8; }
    }

    const std::vector<uint32_t>& remapFor(int colPos, const Dict* d) {  // getOrBuildRemap :120-134
        auto& m = remaps[colPos];
        auto it = m.find(d);
        if (it != m.end()) return it->second;
        std::vector<uint32_t> r(d->keys.size());
        for (size_t lc = 0; lc < d->keys.size(); lc++) r[lc] = globalDicts[colPos].add(d->keys[lc]);
        return m.emplace(d, std::move(r)).first->second;
    }

    bool codeOverflows() const {  // :139-147
        for (size_t i = 0; i < globalDicts.size(); i++)
            if ((uint64_t)globalDicts[i].keys.size() >= (1ULL << widths[i])) return true;
        return false;
    }

    std::string intKeyToStringKey(uint64_t ik) {  // :166-190
        std::string k;
        Group& g = intGroups[ik];
        for (size_t i = 0; i < groupBy.size(); i++) {
            uint32_t code = (uint32_t)((ik >> shifts[i]) & ((1ULL << widths[i]) - 1));
            if (!g.sample.empty() && g.sample[i].isNull) { k.push_back((char)0); k.push_back((char)0xFF); }
            else {
                const std::string& s = globalDicts[i].keys[code];
                k.push_back((char)0x02);
                uint32_t len = (uint32_t)s.size();
                k.append((const char*)&len, 4);
                k += s;
                k.push_back((char)0xFF);
            }
        }
        return k;
    }

    void materializeToStringMaps() {  // :153-164
        for (uint64_t ik : intKeys) {
            std::string sk = intKeyToStringKey(ik);
            keys.push_back(sk);
            groups[sk] = std::move(intGroups[ik]);
        }
        intKeys.clear();
        intGroups.clear();
    }

    // accumulate (aggregate.go:361-559)
    void accumulate(const Batch& b, const std::vector<const Vec*>& av) {
        int rows = b.rows();
        if (groupBy.empty()) {  // accumulateDirect (aggregate.go:567-745)
            const std::string key;
            auto it = groups.find(key);
            if (it == groups.end()) {
                it = groups.emplace(key, newGroup()).first;
                keys.push_back(key);
            }
            Group& g = it->second;
            for (size_t j = 0; j < aggs.size(); j++) {
                const AggSpec& a = aggs[j];
                const Vec* v = av[j];
                if (a.kind == VEXQ_AGG_COUNT && a.star) { g.accs[j] += rows; g.nonNull[j] += rows; continue; }
                if (a.kind == VEXQ_AGG_SUM && a.accum == VEXQ_TYPE_FLOAT64) {
                    double cur = bitsToF(g.accs[j]);
                    for (int ri = 0; ri < rows; ri++) {
                        int r = b.rowAt(ri);
                        if (!v->isNull(r)) { cur += v->f64[r]; g.nonNull[j]++; if (trackExact) g.exact[j].add(v->f64[r]); }
                    }
                    g.accs[j] = fToBits(cur);
                    continue;
                }
                for (int ri = 0; ri < rows; ri++) {
                    int r = b.rowAt(ri);
                    // the remaining kinds fold exactly as foldRow does, one agg at a time
                    const AggSpec& aa = a;
                    const Vec* vv = v;
                    switch (aa.kind) {
                        case VEXQ_AGG_COUNT: if (!vv->isNull(r)) { g.accs[j]++; g.nonNull[j]++; } break;
                        case VEXQ_AGG_COUNT_DISTINCT: foldDistinct(g, j, vv, r); break;
                        case VEXQ_AGG_SUM:
                            if (!vv->isNull(r)) { g.accs[j] = (int64_t)((uint64_t)g.accs[j] + (uint64_t)extractInt64(*vv, r)); g.nonNull[j]++; }
                            break;
                        case VEXQ_AGG_AVG:
                            if (!vv->isNull(r)) {
                                double x = vv->type == VEXQ_TYPE_FLOAT64 ? vv->f64[r] : (double)extractInt64(*vv, r);
                                g.accs[j] = fToBits(bitsToF(g.accs[j]) + x);
                                g.nonNull[j]++;
                                if (trackExact) g.exact[j].add(x);
                            }
                            break;
                        case VEXQ_AGG_MIN:
                        case VEXQ_AGG_MAX: {
                            if (vv->isNull(r)) break;
                            bool less = aa.kind == VEXQ_AGG_MIN;
                            if (aa.accum == VEXQ_TYPE_STRING) {
                                minMaxString(g.strs, j, vv->str(r), g.nonNull[j] > 0, less);
                                g.nonNull[j]++;
                                break;
                            }
                            if (aa.accum == VEXQ_TYPE_FLOAT64) {
                                double cur = bitsToF(g.accs[j]), f = vv->f64[r];
                                if ((less && f < cur) || (!less && f > cur)) g.accs[j] = fToBits(f);
                            } else {
                                int64_t val = extractInt64(*vv, r);
                                if ((less && val < g.accs[j]) || (!less && val > g.accs[j])) g.accs[j] = val;
                            }
                            g.nonNull[j]++;
                            break;
                        }
                    }
                }
            }
            return;
        }
        if (!ikDecided) {  // canUseIntKey (agg_intkey.go:104-116); COUNT(DISTINCT) turns it off (aggregate.go:396-399)
            ikDecided = true;
            bool ok = groupBy.size() <= 8 && !hasDistinct();
            for (int c : groupBy) if (b.cols[c]->type != VEXQ_TYPE_STRING || !b.cols[c]->dict) ok = false;
            if (ok) { ikEnabled = true; initIntKey((int)groupBy.size()); }
        }
        if (ikEnabled) {  // accumulateIntKey (agg_intkey.go:206-290)
            size_t ng = groupBy.size();
            const Vec* sv[8];
            const std::vector<uint32_t>* rm[8];
            for (size_t i = 0; i < ng; i++) {
                sv[i] = b.cols[groupBy[i]];
                rm[i] = &remapFor((int)i, sv[i]->dict);
            }
            if (codeOverflows()) {
                ikEnabled = false;
                if (!intKeys.empty()) materializeToStringMaps();
                for (int ri = 0; ri < rows; ri++) { int r = b.rowAt(ri); accumulateOneRow(buildKey(b, r), b, r, av); }
                return;
            }
            for (int ri = 0; ri < rows; ri++) {
                int r = b.rowAt(ri);
                bool hasNull = false;
                for (size_t i = 0; i < ng; i++) if (sv[i]->isNull(r)) { hasNull = true; break; }
                if (hasNull) { accumulateOneRow(buildKey(b, r), b, r, av); continue; }
                uint64_t key = 0;
                for (size_t i = 0; i < ng; i++) key |= (uint64_t)(*rm[i])[sv[i]->codes[r]] << shifts[i];
                auto it = intGroups.find(key);
                if (it == intGroups.end()) {
                    Group g = newGroup();
                    g.sample.resize(ng);
                    for (size_t i = 0; i < ng; i++) g.sample[i].str = sv[i]->str(r);
                    it = intGroups.emplace(key, std::move(g)).first;
                    intKeys.push_back(key);
                }
                foldRow(it->second, av, r);
            }
            return;
        }
        for (int ri = 0; ri < rows; ri++) { int r = b.rowAt(ri); accumulateOneRow(buildKey(b, r), b, r, av); }
    }

    void finish() {  // consumeAll tail (aggregate.go:339-343)
        if (ikEnabled && !intKeys.empty()) materializeToStringMaps();
    }
};

// mergePartialAgg (exec/parallel.go:237-314)
void mergePartialAgg(HashAgg& dst, HashAgg& src) {
    for (const std::string& key : src.keys) {
        Group& s = src.groups[key];
        auto it = dst.groups.find(key);
        if (it == dst.groups.end()) {
            dst.groups.emplace(key, s);
            dst.keys.push_back(key);
            continue;
        }
        Group& d = it->second;
        for (size_t j = 0; j < dst.aggs.size(); j++) {
            const AggSpec& a = dst.aggs[j];
            switch (a.kind) {
                case VEXQ_AGG_COUNT: d.accs[j] = (int64_t)((uint64_t)d.accs[j] + (uint64_t)s.accs[j]); break;
                case VEXQ_AGG_SUM:
                case VEXQ_AGG_AVG:
                    if (a.accum == VEXQ_TYPE_FLOAT64) d.accs[j] = fToBits(bitsToF(d.accs[j]) + bitsToF(s.accs[j]));
                    else d.accs[j] = (int64_t)((uint64_t)d.accs[j] + (uint64_t)s.accs[j]);
                    break;
                case VEXQ_AGG_MIN:
                case VEXQ_AGG_MAX: {
                    bool less = a.kind == VEXQ_AGG_MIN;
                    if (a.accum == VEXQ_TYPE_STRING) {
                        if (s.nonNull[j] == 0) break;
                        HashAgg::minMaxString(d.strs, j, s.strs[j], d.nonNull[j] > 0, less);
                        break;
                    }
                    if (a.accum == VEXQ_TYPE_FLOAT64) {
                        double df = bitsToF(d.accs[j]), sf = bitsToF(s.accs[j]);
                        if ((less && sf < df) || (!less && sf > df)) d.accs[j] = s.accs[j];
                    } else if ((less && s.accs[j] < d.accs[j]) || (!less && s.accs[j] > d.accs[j])) {
                        d.accs[j] = s.accs[j];
                    }
                    break;
                }
            }
        }
        for (size_t j = 0; j < d.nonNull.size(); j++) d.nonNull[j] += s.nonNull[j];
    }
}

// ---- results ---------------------------------------------------------------------
struct OutCol {
    std::string name;
    int type;
    std::vector<int64_t> bits;
    std::vector<uint8_t> valid;
    std::vector<std::string> strs;
    std::vector<double> exact;
};

}  // namespace

struct ref_table_s {
    Table t;
};
struct ref_result_s {
    std::vector<OutCol> cols;
    int64_t rows = 0;
};

namespace {

// buildOutputBatch (aggregate.go:780-955) over all groups at once, and
// buildEmptyGlobalResult (:961-982).
ref_result_s* buildOutput(HashAgg& h, const std::vector<int>& gbOutTypes) {
    auto* res = new ref_result_s;
    size_t n = h.keys.size();
    bool emptyGlobal = n == 0 && h.groupBy.empty();
    size_t rows = emptyGlobal ? 1 : n;
    res->rows = (int64_t)rows;
    for (size_t gi = 0; gi < h.groupBy.size(); gi++) {
        OutCol c;
        c.name = "gb" + std::to_string(gi);
        c.type = gbOutTypes[gi];
        c.bits.assign(rows, 0);
        c.valid.assign(rows, 0);
        c.strs.assign(rows, "");
        c.exact.assign(rows, NAN);
        for (size_t i = 0; i < n; i++) {
            const Group& g = h.groups[h.keys[i]];
            const GroupByVal& s = g.sample[gi];
            if (s.isNull) continue;
            c.valid[i] = 1;
            if (c.type == VEXQ_TYPE_STRING) c.strs[i] = s.str;
            else if (c.type == VEXQ_TYPE_DATE) c.bits[i] = (int64_t)(int32_t)s.bits;
            else if (c.type == VEXQ_TYPE_BOOL) c.bits[i] = s.bits != 0;
            else c.bits[i] = (int64_t)s.bits;
        }
        res->cols.push_back(std::move(c));
    }
    for (size_t j = 0; j < h.aggs.size(); j++) {
        const AggSpec& a = h.aggs[j];
        OutCol c;
        c.name = a.name;
        c.bits.assign(rows, 0);
        c.valid.assign(rows, 0);
        c.strs.assign(rows, "");
        c.exact.assign(rows, NAN);
        switch (a.kind) {
            case VEXQ_AGG_COUNT:
            case VEXQ_AGG_COUNT_DISTINCT: c.type = VEXQ_TYPE_INT64; break;
            case VEXQ_AGG_SUM: c.type = a.accum == VEXQ_TYPE_FLOAT64 ? VEXQ_TYPE_FLOAT64 : VEXQ_TYPE_INT64; break;
            case VEXQ_AGG_AVG: c.type = VEXQ_TYPE_FLOAT64; break;
            default: c.type = a.outType; break;
        }
        if (emptyGlobal) {
            if (a.kind == VEXQ_AGG_COUNT || a.kind == VEXQ_AGG_COUNT_DISTINCT) c.valid[0] = 1;  // COUNT → 0, others NULL
            res->cols.push_back(std::move(c));
            continue;
        }
        for (size_t i = 0; i < n; i++) {
            const Group& g = h.groups[h.keys[i]];
            int64_t nn = g.nonNull[j];
            switch (a.kind) {
                case VEXQ_AGG_COUNT: c.valid[i] = 1; c.bits[i] = g.accs[j]; break;
                case VEXQ_AGG_COUNT_DISTINCT:  // the set's size, never NULL (aggregate.go:810-823)
                    c.valid[i] = 1;
                    c.bits[i] = g.dints.empty() ? 0 : (int64_t)(g.dints[j].size() + g.dstrs[j].size());
                    break;
                case VEXQ_AGG_SUM:
                    if (nn == 0) break;
                    c.valid[i] = 1;
                    c.bits[i] = g.accs[j];
                    if (!g.exact.empty() && a.accum == VEXQ_TYPE_FLOAT64) c.exact[i] = g.exact[j].value();
                    break;
                case VEXQ_AGG_AVG:
                    if (nn == 0) break;
                    c.valid[i] = 1;
                    c.bits[i] = fToBits(bitsToF(g.accs[j]) / (double)nn);
                    if (!g.exact.empty()) c.exact[i] = g.exact[j].value() / (double)nn;
                    break;
                default:
                    if (nn == 0) break;
                    c.valid[i] = 1;
                    if (c.type == VEXQ_TYPE_STRING) c.strs[i] = g.strs[j];
                    else if (c.type == VEXQ_TYPE_DATE) c.bits[i] = (int64_t)(int32_t)g.accs[j];
                    else if (c.type == VEXQ_TYPE_BOOL) c.bits[i] = g.accs[j] != 0;
                    else c.bits[i] = g.accs[j];
                    break;
            }
        }
        res->cols.push_back(std::move(c));
    }
    return res;
}

// ExternalSort.less (exec/sort.go:130-163) + Limit (exec/limit.go:20-50)
void applyOrder(ref_result_s* r, const vexq_order_desc& o) {
    if (o.sort_col >= 0) {
        if (o.sort_col >= (int)r->cols.size()) throw Error("ORDER BY column out of range");
        const OutCol& k = r->cols[o.sort_col];
        std::vector<int64_t> idx(r->rows);
        for (int64_t i = 0; i < r->rows; i++) idx[i] = i;
        std::stable_sort(idx.begin(), idx.end(), [&](int64_t a, int64_t b) {
            bool aN = !k.valid[a], bN = !k.valid[b];
            if (aN && bN) return false;
            if (aN) return true;
            if (bN) return false;
            if (k.type == VEXQ_TYPE_STRING) {
                if (k.strs[a] == k.strs[b]) return false;
                return o.descending ? k.strs[a] > k.strs[b] : k.strs[a] < k.strs[b];
            }
            if (k.bits[a] == k.bits[b]) return false;
            return o.descending ? k.bits[a] > k.bits[b] : k.bits[a] < k.bits[b];
        });
        for (auto& c : r->cols) {
            OutCol n = c;
            for (int64_t i = 0; i < r->rows; i++) {
                n.bits[i] = c.bits[idx[i]];
                n.valid[i] = c.valid[idx[i]];
                n.strs[i] = c.strs[idx[i]];
                n.exact[i] = c.exact[idx[i]];
            }
            c = std::move(n);
        }
    }
    if (o.limit >= 0 && o.limit < r->rows) {
        for (auto& c : r->cols) {
            c.bits.resize(o.limit);
            c.valid.resize(o.limit);
            c.strs.resize(o.limit);
            c.exact.resize(o.limit);
        }
        r->rows = o.limit;
    }
}

// resolveAggConfig (planner/physical.go:198-259) for agg descriptors whose
// inputs are expressions over `schema`.
struct AggPlan {
    std::vector<AggSpec> specs;
    std::vector<XP> inputs;  // null for COUNT(*)
    std::vector<bool> plain; // input is a bare column reference
    std::vector<int> gb;
    std::vector<int> gbTypes;
};

AggPlan resolveAggs(const Nodes& N, const vexq_agg_desc* aggs, int naggs, const int32_t* gb, int ngb,
                    const Schema& s) {
    AggPlan p;
    for (int i = 0; i < ngb; i++) {
        if (gb[i] < 0 || gb[i] >= (int)s.types.size()) throw Error("GROUP BY column out of range");
        p.gb.push_back(gb[i]);
        p.gbTypes.push_back(s.types[gb[i]]);
    }
    for (int j = 0; j < naggs; j++) {
        AggSpec a;
        a.kind = aggs[j].kind;
        a.name = aggs[j].out_name ? aggs[j].out_name : "";
        if (a.kind < VEXQ_AGG_COUNT || a.kind > VEXQ_AGG_COUNT_DISTINCT) throw Error("unknown aggregate kind");
        a.star = aggs[j].input < 0;
        if (a.star && a.kind != VEXQ_AGG_COUNT) throw Error("aggregate column not found");
        XP in;
        if (!a.star) {
            in = build(N, aggs[j].input, s);
            a.srcType = in->type;
            p.plain.push_back(N.at(aggs[j].input).kind == VEXQ_E_COLUMN);
        } else {
            a.srcType = VEXQ_TYPE_INT64;
            p.plain.push_back(true);
        }
        a.accum = a.kind == VEXQ_AGG_COUNT || a.kind == VEXQ_AGG_COUNT_DISTINCT ? VEXQ_TYPE_INT64
                                                                                : accumTypeFor(a.kind, a.srcType);
        switch (a.kind) {
            case VEXQ_AGG_COUNT:
            case VEXQ_AGG_COUNT_DISTINCT: a.outType = VEXQ_TYPE_INT64; break;
            case VEXQ_AGG_AVG: a.outType = VEXQ_TYPE_FLOAT64; break;
            default: a.outType = a.srcType; break;
        }
        p.specs.push_back(a);
        p.inputs.push_back(std::move(in));
    }
    return p;
}

// Per-pipeline state: predicate + aggregate input expressions (each worker
// owns its own copy, as each goroutine owns its pipeline).
struct AggPipeline {
    XP pred;
    AggPlan plan;
    HashAgg ha;
    std::vector<const Vec*> av;
    std::vector<Vec> mat;  // Project.materialize output per agg input
    std::vector<Vec> gbm;  // materialised group-by columns
};

AggPipeline makeAggPipeline(const Nodes& N, const vexq_agg_plan_desc* d, const Schema& s, bool exact) {
    AggPipeline p;
    if (d->predicate >= 0) {
        p.pred = build(N, d->predicate, s);
        if (p.pred->type != VEXQ_TYPE_BOOL) throw Error("filter predicate must return BOOL");
    }
    p.plan = resolveAggs(N, d->aggs, d->naggs, d->group_by, d->ngroup_by, s);
    if (d->naggs == 0 && d->ngroup_by == 0) throw Error("hash aggregate: no group-by columns or aggregate expressions");
    p.ha.groupBy = p.plan.gb;
    p.ha.aggs = p.plan.specs;
    p.ha.trackExact = exact;
    p.ha.initMaps();
    p.av.assign(d->naggs, nullptr);
    p.mat.resize(d->naggs);
    p.gbm.resize(p.plan.gb.size());
    return p;
}

// BoolToSelVecInto (expr.go:1545-1564)
void selectInto(Batch& b, const Vec* bv) {
    std::vector<uint16_t> out;
    out.reserve(bv->n);
    if (!b.has_sel) {
        for (int i = 0; i < bv->n; i++) if (bv->valid[i] && bv->bits[i]) out.push_back((uint16_t)i);
    } else {
        for (uint16_t i : b.sel) if (bv->valid[i] && bv->bits[i]) out.push_back(i);
    }
    b.sel.swap(out);
    b.has_sel = true;
    b.length = (int)b.sel.size();
}

// Project.materialize (exec/project.go:128-196)
void materialize(const Vec& src, const std::vector<uint16_t>& sel, Vec& out) {
    int n = (int)sel.size();
    out.resize(src.type, n);
    out.dict = src.dict;
    out.owned = src.owned;
    for (int i = 0; i < n; i++) {
        int r = sel[i];
        out.valid[i] = src.valid[r];
        switch (src.type) {
            case VEXQ_TYPE_INT64: out.i64[i] = src.i64[r]; break;
            case VEXQ_TYPE_FLOAT64: out.f64[i] = src.f64[r]; break;
            case VEXQ_TYPE_DATE: out.i32[i] = src.i32[r]; break;
            case VEXQ_TYPE_STRING: out.codes[i] = src.codes[r]; break;
            case VEXQ_TYPE_BOOL: out.bits[i] = src.bits[r]; break;
        }
    }
}

// Filter.Next → Project.Next → HashAggregate.accumulate for one batch.
void runBatch(AggPipeline& p, Batch& b) {
    if (p.pred) {  // Filter.Next (filter.go:49-78)
        const Vec* bv = eval(p.pred.get(), b);
        selectInto(b, bv);
        if (b.sel.empty()) return;
    }
    // Pre-projection: expression aggregates are evaluated over physical rows
    // and compacted by the selection vector (project.go:64-110). Plain columns
    // are read through the selection vector directly; the visited rows and
    // their order are the same.
    bool anyComplex = false;
    for (size_t j = 0; j < p.plan.specs.size(); j++) if (!p.plan.plain[j]) anyComplex = true;
    if (!anyComplex) {
        for (size_t j = 0; j < p.plan.specs.size(); j++)
            p.av[j] = p.plan.specs[j].star ? b.cols.empty() ? nullptr : b.cols[0] : eval(p.plan.inputs[j].get(), b);
        p.ha.accumulate(b, p.av);
        return;
    }
    // Materialise every column the aggregate reads into a compacted batch.
    Batch cb;
    std::vector<Vec>& gbm = p.gbm;
    cb.cols.assign(b.cols.size(), nullptr);
    if (b.has_sel) {
        for (size_t gi = 0; gi < p.plan.gb.size(); gi++) {
            materialize(*b.cols[p.plan.gb[gi]], b.sel, gbm[gi]);
            cb.cols[p.plan.gb[gi]] = &gbm[gi];
        }
    } else {
        for (int gbc : p.plan.gb) cb.cols[gbc] = b.cols[gbc];
    }
    for (size_t j = 0; j < p.plan.specs.size(); j++) {
        if (p.plan.specs[j].star) { p.av[j] = nullptr; continue; }
        const Vec* raw = eval(p.plan.inputs[j].get(), b);
        if (b.has_sel) { materialize(*raw, b.sel, p.mat[j]); p.av[j] = &p.mat[j]; }
        else { p.mat[j] = *raw; p.av[j] = &p.mat[j]; }
    }
    cb.length = b.rows();
    cb.phys = cb.length;
    cb.has_sel = false;
    p.ha.accumulate(cb, p.av);
}

Schema tableSchema(const Table& t) {
    Schema s;
    for (auto& c : t.cols) s.types.push_back(c.type);
    return s;
}

// Scans row groups [rgs, rge) of t with zone pruning, feeding runBatch.
void scanRange(const Table& t, const Nodes& N, int predRoot, int rgs, int rge, AggPipeline& p, Scan& sc) {
    Batch b;
    for (int rg = rgs; rg < rge; rg++) {
        if (predRoot >= 0 && !zoneEval(N, predRoot, t, rg)) continue;  // scan.go:212-215
        for (int64_t s = t.rgStart(rg); s < t.rgEnd(rg); s += kBlockRows) {
            int n = (int)std::min<int64_t>(kBlockRows, t.rgEnd(rg) - s);
            sc.load(rg, s, n, b);
            runBatch(p, b);
        }
    }
}

ref_result_s* runAgg(const Table& t, const vexq_agg_plan_desc* d, int rgs, int rge, int workers) {
    Nodes N{d->nodes, d->nnodes, d->children, d->nchildren};
    Schema s = tableSchema(t);
    std::vector<char> need(t.cols.size(), 0);
    collectCols(N, d->predicate, need);
    for (int i = 0; i < d->ngroup_by; i++) if (d->group_by[i] >= 0 && d->group_by[i] < (int)need.size()) need[d->group_by[i]] = 1;
    for (int j = 0; j < d->naggs; j++) collectCols(N, d->aggs[j].input, need);
    // COUNT(DISTINCT) runs serially: partial distinct counts cannot be summed
    // (planner/parallel.go:218-228)
    for (int j = 0; j < d->naggs; j++)
        if (d->aggs[j].kind == VEXQ_AGG_COUNT_DISTINCT) workers = 0;
    if (workers <= 0) {  // planner.Physical: one pipeline, strict row order
        AggPipeline p = makeAggPipeline(N, d, s, true);
        Scan sc(&t, need);
        scanRange(t, N, d->predicate, rgs, rge, p, sc);
        p.ha.finish();
        ref_result_s* r = buildOutput(p.ha, p.plan.gbTypes);
        applyOrder(r, d->order);
        return r;
    }
    // ParallelHashAggregate.setup (exec/parallel.go:124-210)
    int total = rge - rgs;
    if (workers > total && total > 0) workers = total;
    if (workers < 1) workers = 1;
    std::atomic<int64_t> next{rgs};
    std::vector<AggPipeline> parts;
    for (int w = 0; w < workers; w++) parts.push_back(makeAggPipeline(N, d, s, false));
    std::vector<std::thread> th;
    std::vector<std::string> errs(workers);
    for (int w = 0; w < workers; w++) {
        th.emplace_back([&, w]() {
            try {
                Scan sc(&t, need);
                for (;;) {
                    int64_t start = next.fetch_add(1);  // morselQueue.claim (parallel.go:26-36)
                    if (start >= rge) break;
                    scanRange(t, N, d->predicate, (int)start, (int)start + 1, parts[w], sc);
                }
                parts[w].ha.finish();
            } catch (const std::exception& e) {
                errs[w] = e.what();
            }
        });
    }
    for (auto& x : th) x.join();
    for (auto& e : errs) if (!e.empty()) throw Error(e);
    AggPipeline merged = makeAggPipeline(N, d, s, false);
    for (int w = 0; w < workers; w++) mergePartialAgg(merged.ha, parts[w].ha);
    ref_result_s* r = buildOutput(merged.ha, merged.plan.gbTypes);
    applyOrder(r, d->order);
    return r;
}

// ---- join (exec/join.go, exec/join_table.go, exec/parallel_join.go) ------------------

// radixHash (parallel_join.go:91-99): murmur3 fmix64
inline uint64_t radixHash(int64_t key) {
    uint64_t x = (uint64_t)key;
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdULL;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ULL;
    x ^= x >> 33;
    return x;
}

// RadixBitsFor (parallel_join.go:72-81)
int radixBitsFor(int64_t est) {
    if (est < 65536) return 0;
    int bits = 4;
    while (bits < 6 && (int64_t(1) << bits) * 8192 < est) bits++;
    return bits;
}

// rowStore + joinHashTable (join_table.go:111-569): build rows with
// insertion-ordered per-key chains, linear probing on the high hash bits.
struct RowStore {
    int ncols;
    std::vector<int64_t> values;
    std::vector<uint8_t> nulls;
    std::vector<std::string> strs;  // one per (row, col) for string columns
    std::vector<int32_t> next;
    int32_t n = 0;
};

struct JoinTable {
    struct Slot { int64_t key; int32_t head, tail; };
    std::vector<Slot> slots;
    uint64_t mask = 0;
    unsigned shift = 0;
    int keys = 0, growAt = 0, numRow = 0;
    RowStore* store = nullptr;
    static int capacityFor(int k) {  // joinTableCapacity :444-460
        int slots = 8;
        if (k <= 0) return slots;
        int64_t need = ((int64_t)k * 10 + 7 - 1) / 7;
        while (slots < need) slots *= 2;
        return slots;
    }
    void setCapacity(int cap) {
        slots.assign(cap, Slot{0, -1, -1});
        mask = (uint64_t)cap - 1;
        shift = 64 - __builtin_ctzll((uint64_t)cap);
        growAt = cap * 7 / 10;
    }
    void grow() {
        std::vector<Slot> old = slots;
        setCapacity((int)old.size() * 2);
        for (auto& s : old) {
            if (s.head == -1) continue;
            uint64_t i = radixHash(s.key) >> shift;
            while (slots[i].head != -1) i = (i + 1) & mask;
            slots[i] = s;
        }
    }
    void insert(int64_t key, int32_t row) {  // :496-517
        if (keys >= growAt) grow();
        store->next[row] = -1;
        numRow++;
        uint64_t i = radixHash(key) >> shift;
        for (;;) {
            Slot& s = slots[i];
            if (s.head == -1) { s.key = key; s.head = row; s.tail = row; keys++; return; }
            if (s.key == key) { store->next[s.tail] = row; s.tail = row; return; }
            i = (i + 1) & mask;
        }
    }
    int32_t lookup(int64_t key, uint64_t h) const {  // lookupHashed :529-541
        uint64_t i = h >> shift;
        for (;;) {
            const Slot& s = slots[i];
            if (s.head == -1) return -1;
            if (s.key == key) return s.head;
            i = (i + 1) & mask;
        }
    }
};

struct SharedTable {
    RowStore store;
    std::vector<JoinTable> parts;
    uint64_t partMask = 0;
    int numRows = 0;
};

// Drains the build side (Scan → Filter) in row order; forEachBuildRow
// (join.go:200-241) drops NULL keys. The serial radix build and the two-pass
// parallel build (parallel_join.go:235-271, 389-552) yield the same per-key
// chains (row order), so one deterministic construction serves both.
void buildShared(const Table& bt, const Nodes& N, const vexq_join_plan_desc* d, SharedTable& sht) {
    Schema bs = tableSchema(bt);
    XP pred;
    if (d->build_predicate >= 0) pred = build(N, d->build_predicate, bs);
    int nb = (int)bt.cols.size();
    if (d->build_key < 0 || d->build_key >= nb) throw Error("build key out of range");
    RowStore& st = sht.store;
    st.ncols = nb;
    int bits = d->radix_bits >= 0 ? std::min(d->radix_bits, 12) : radixBitsFor(bt.nrows);
    int nparts = 1 << bits;
    sht.partMask = (uint64_t)(nparts - 1);
    std::vector<std::vector<std::pair<int64_t, int32_t>>> byPart(nparts);
    Scan sc(&bt);
    Batch b;
    for (int rg = 0; rg < bt.n_rg; rg++) {
        if (d->build_predicate >= 0 && !zoneEval(N, d->build_predicate, bt, rg)) continue;
        for (int64_t s = bt.rgStart(rg); s < bt.rgEnd(rg); s += kBlockRows) {
            int n = (int)std::min<int64_t>(kBlockRows, bt.rgEnd(rg) - s);
            sc.load(rg, s, n, b);
            if (pred) {
                selectInto(b, eval(pred.get(), b));
                if (b.sel.empty()) continue;
            }
            const Vec* kv = b.cols[d->build_key];
            for (int ri = 0; ri < b.rows(); ri++) {
                int r = b.rowAt(ri);
                if (kv->isNull(r)) continue;
                int64_t key = extractInt64(*kv, r);
                int32_t row = st.n++;
                for (int c = 0; c < nb; c++) {
                    const Vec* v = b.cols[c];
                    bool isn = v->isNull(r);
                    st.nulls.push_back(isn);
                    st.values.push_back(isn || v->type == VEXQ_TYPE_STRING ? 0 : extractInt64(*v, r));
                    st.strs.push_back(!isn && v->type == VEXQ_TYPE_STRING ? v->str(r) : std::string());
                }
                st.next.push_back(-1);
                uint64_t p = nparts > 1 ? (radixHash(key) & sht.partMask) : 0;
                byPart[p].push_back({key, row});
            }
        }
    }
    // Pass 2: partition tables presized from exact counts; rows inserted in
    // row order within each partition.
    sht.parts.resize(nparts);
    for (int p = 0; p < nparts; p++) {
        sht.parts[p].store = &st;
        sht.parts[p].setCapacity(JoinTable::capacityFor((int)byPart[p].size()));
        for (auto& kr : byPart[p]) sht.parts[p].insert(kr.first, kr.second);
    }
    sht.numRows = st.n;
}

int sharedKeys(const SharedTable& s) {
    int k = 0;
    for (auto& p : s.parts) k += p.keys;
    return k;
}

// HashJoin.Next probe + emitMatches (join.go:84-155, 243-403): for each
// probe batch, every match in probe (SelVec) order then chain order, emitted
// in ≤1024-row joined batches (build columns, then probe columns).
struct JoinedBatcher {
    int nb, np;
    std::vector<Vec> vecs;
    std::vector<const Vec*> ptrs;
    JoinedBatcher(int b, int p) : nb(b), np(p), vecs(b + p) { for (auto& v : vecs) ptrs.push_back(&v); }
    void fill(const SharedTable& sht, const Table& bt, const Batch& pb,
              const std::vector<std::pair<int32_t, int32_t>>& m, size_t s, size_t e, Batch& out) {
        int n = (int)(e - s);
        const RowStore& st = sht.store;
        for (int c = 0; c < nb; c++) {
            Vec& v = vecs[c];
            int t = bt.cols[c].type;
            v.resize(t, n);
            v.owned.reset();
            v.dict = nullptr;
            std::shared_ptr<Dict> db;
            if (t == VEXQ_TYPE_STRING) db = std::make_shared<Dict>();
            for (int i = 0; i < n; i++) {
                int32_t br = m[s + i].first;
                if (st.nulls[(size_t)br * nb + c]) continue;
                v.valid[i] = 1;
                int64_t val = st.values[(size_t)br * nb + c];
                switch (t) {
                    case VEXQ_TYPE_INT64: v.i64[i] = val; break;
                    case VEXQ_TYPE_FLOAT64: v.f64[i] = bitsToF(val); break;
                    case VEXQ_TYPE_DATE: v.i32[i] = (int32_t)val; break;
                    case VEXQ_TYPE_BOOL: v.bits[i] = val != 0; break;
                    case VEXQ_TYPE_STRING: v.codes[i] = db->add(st.strs[(size_t)br * nb + c]); break;
                }
            }
            if (db) { v.owned = db; v.dict = db.get(); }
        }
        for (int c = 0; c < np; c++) {
            Vec& v = vecs[nb + c];
            const Vec* src = pb.cols[c];
            v.resize(src->type, n);
            v.owned.reset();
            v.dict = src->dict;
            for (int i = 0; i < n; i++) {
                int pr = m[s + i].second;
                if (src->isNull(pr)) continue;
                v.valid[i] = 1;
                switch (src->type) {
                    case VEXQ_TYPE_INT64: v.i64[i] = src->i64[pr]; break;
                    case VEXQ_TYPE_FLOAT64: v.f64[i] = src->f64[pr]; break;
                    case VEXQ_TYPE_DATE: v.i32[i] = src->i32[pr]; break;
                    case VEXQ_TYPE_BOOL: v.bits[i] = src->bits[pr]; break;
                    case VEXQ_TYPE_STRING: v.codes[i] = src->codes[pr]; break;
                }
            }
        }
        out.cols = ptrs;
        out.length = n;
        out.phys = n;
        out.has_sel = false;
        out.sel.clear();
    }
};

struct JoinPipeline {
    XP probePred;
    AggPipeline above;  // residual filter + aggregate over the joined schema
};

JoinPipeline makeJoinPipeline(const Nodes& N, const vexq_join_plan_desc* d, const Schema& ps, const Schema& js,
                              bool exact) {
    JoinPipeline jp;
    if (d->probe_predicate >= 0) jp.probePred = build(N, d->probe_predicate, ps);
    vexq_agg_plan_desc ad{};
    ad.nodes = d->nodes;
    ad.nnodes = d->nnodes;
    ad.children = d->children;
    ad.nchildren = d->nchildren;
    ad.predicate = d->residual;
    ad.group_by = d->group_by;
    ad.ngroup_by = d->ngroup_by;
    ad.aggs = d->aggs;
    ad.naggs = d->naggs;
    jp.above = makeAggPipeline(N, &ad, js, exact);
    return jp;
}

void probeRange(const Table& pt, const Table& bt, const SharedTable& sht, const Nodes& N,
                const vexq_join_plan_desc* d, int rgs, int rge, JoinPipeline& jp, Scan& sc, JoinedBatcher& jb) {
    Batch b, out;
    std::vector<std::pair<int32_t, int32_t>> matches;
    for (int rg = rgs; rg < rge; rg++) {
        if (d->probe_predicate >= 0 && !zoneEval(N, d->probe_predicate, pt, rg)) continue;
        for (int64_t s = pt.rgStart(rg); s < pt.rgEnd(rg); s += kBlockRows) {
            int n = (int)std::min<int64_t>(kBlockRows, pt.rgEnd(rg) - s);
            sc.load(rg, s, n, b);
            if (jp.probePred) {
                selectInto(b, eval(jp.probePred.get(), b));
                if (b.sel.empty()) continue;
            }
            matches.clear();
            const Vec* kv = b.cols[d->probe_key];
            for (int ri = 0; ri < b.rows(); ri++) {
                int r = b.rowAt(ri);
                if (kv->isNull(r)) continue;
                int64_t key = extractInt64(*kv, r);
                uint64_t h = radixHash(key);
                const JoinTable& tbl = sht.parts[h & sht.partMask];
                for (int32_t bi = tbl.lookup(key, h); bi != -1; bi = sht.store.next[bi]) matches.push_back({bi, r});
            }
            for (size_t ms = 0; ms < matches.size(); ms += kBlockRows) {
                size_t me = std::min(matches.size(), ms + kBlockRows);
                jb.fill(sht, bt, b, matches, ms, me, out);
                runBatch(jp.above, out);
            }
        }
    }
}

ref_result_s* runJoin(const Table& bt, const Table& pt, const vexq_join_plan_desc* d, int workers) {
    Nodes N{d->nodes, d->nnodes, d->children, d->nchildren};
    Schema bs = tableSchema(bt), ps = tableSchema(pt), js;
    js.types = bs.types;
    js.types.insert(js.types.end(), ps.types.begin(), ps.types.end());
    if (d->probe_key < 0 || d->probe_key >= (int)pt.cols.size()) throw Error("probe key out of range");
    SharedTable sht;
    buildShared(bt, N, d, sht);
    int nb = (int)bt.cols.size(), np = (int)pt.cols.size();
    if (workers <= 0) {
        JoinPipeline jp = makeJoinPipeline(N, d, ps, js, true);
        if (sharedKeys(sht) > 0) {
            Scan sc(&pt);
            JoinedBatcher jb(nb, np);
            probeRange(pt, bt, sht, N, d, 0, pt.n_rg, jp, sc, jb);
        }
        jp.above.ha.finish();
        ref_result_s* r = buildOutput(jp.above.ha, jp.above.plan.gbTypes);
        applyOrder(r, d->order);
        return r;
    }
    // runMorselAggWorkers (parallel_join.go:911-988)
    std::vector<JoinPipeline> parts;
    int w = std::max(1, std::min(workers, pt.n_rg));
    for (int i = 0; i < w; i++) parts.push_back(makeJoinPipeline(N, d, ps, js, false));
    if (sharedKeys(sht) > 0 && pt.n_rg > 0) {
        std::atomic<int64_t> next{0};
        std::vector<std::thread> th;
        std::vector<std::string> errs(w);
        for (int i = 0; i < w; i++) {
            th.emplace_back([&, i]() {
                try {
                    Scan sc(&pt);
                    JoinedBatcher jb(nb, np);
                    for (;;) {
                        int64_t st = next.fetch_add(1);
                        if (st >= pt.n_rg) break;
                        probeRange(pt, bt, sht, N, d, (int)st, (int)st + 1, parts[i], sc, jb);
                    }
                    parts[i].above.ha.finish();
                } catch (const std::exception& e) {
                    errs[i] = e.what();
                }
            });
        }
        for (auto& x : th) x.join();
        for (auto& e : errs) if (!e.empty()) throw Error(e);
    }
    JoinPipeline merged = makeJoinPipeline(N, d, ps, js, false);
    for (auto& p : parts) mergePartialAgg(merged.above.ha, p.above.ha);
    ref_result_s* r = buildOutput(merged.above.ha, merged.above.plan.gbTypes);
    applyOrder(r, d->order);
    return r;
}

template <class F>
int32_t guarded(F&& f) {
    try {
        g_err.clear();
        return f();
    } catch (const std::exception& e) {
        g_err = e.what();
        return VEXQ_EINVAL;
    }
}

}  // namespace

extern "C" {

const char* ref_last_error(void) { return g_err.c_str(); }

// The radix-partition choice and partition index of the partitioned join
// (RadixBitsFor and radixPart, parallel_join.go:72-109), for the tests that
// pin them on the reference's own cases.
int32_t ref_radix_bits_for(int64_t est_rows) { return radixBitsFor(est_rows); }
int32_t ref_radix_part(int64_t key, uint64_t mask) { return mask == 0 ? 0 : (int32_t)(radixHash(key) & mask); }

int32_t ref_table_new(const vexq_column_desc* cols, int32_t ncols, int64_t nrows, int32_t rg_rows, ref_table_t* out) {
    return guarded([&]() -> int32_t {
        auto* h = new ref_table_s;
        Table& t = h->t;
        t.nrows = nrows;
        t.rg_rows = rg_rows > 0 ? rg_rows : 65536;
        t.n_rg = (int)((nrows + t.rg_rows - 1) / t.rg_rows);
        for (int c = 0; c < ncols; c++) {
            const vexq_column_desc& d = cols[c];
            Column col;
            col.name = d.name ? d.name : "";
            col.type = d.type;
            col.valid.assign(nrows, 1);
            if (d.validity) {
                col.nullable = true;
                for (int64_t r = 0; r < nrows; r++) col.valid[r] = (d.validity[r >> 3] >> (r & 7)) & 1;
            }
            switch (d.type) {
                case VEXQ_TYPE_INT64: col.i64.assign((const int64_t*)d.values, (const int64_t*)d.values + nrows); break;
                case VEXQ_TYPE_FLOAT64: col.f64.assign((const double*)d.values, (const double*)d.values + nrows); break;
                case VEXQ_TYPE_DATE: col.i32.assign((const int32_t*)d.values, (const int32_t*)d.values + nrows); break;
                case VEXQ_TYPE_BOOL: col.b8.assign((const uint8_t*)d.values, (const uint8_t*)d.values + nrows); break;
                case VEXQ_TYPE_STRING: {
                    col.codes.assign((const uint32_t*)d.values, (const uint32_t*)d.values + nrows);
                    if (!d.dict_str_off || !d.dict_bytes) throw Error("string column without dictionaries");
                    if (!d.dict_rg_first) {  // one table-wide dictionary: codes are global
                        auto dict = std::make_shared<Dict>();
                        uint32_t ne = (uint32_t)d.dict_entries;
                        for (int64_t r = 0; r < nrows; r++)
                            if (col.valid[r] && col.codes[r] >= ne) throw Error("dictionary code out of range");
                        for (uint32_t e = 0; e < ne; e++)
                            dict->add(std::string(d.dict_bytes + d.dict_str_off[e], d.dict_str_off[e + 1] - d.dict_str_off[e]));
                        for (int rg = 0; rg < t.n_rg; rg++) col.dicts.push_back(dict);
                        break;
                    }
                    for (int rg = 0; rg < t.n_rg; rg++) {
                        auto dict = std::make_shared<Dict>();
                        for (uint32_t e = d.dict_rg_first[rg]; e < d.dict_rg_first[rg + 1]; e++)
                            dict->add(std::string(d.dict_bytes + d.dict_str_off[e], d.dict_str_off[e + 1] - d.dict_str_off[e]));
                        // codes must index this row group's dictionary
                        for (int64_t r = t.rgStart(rg); r < t.rgEnd(rg); r++)
                            if (col.valid[r] && col.codes[r] >= dict->keys.size()) throw Error("dictionary code out of range");
                        col.dicts.push_back(std::move(dict));
                    }
                    break;
                }
                default: throw Error("unknown column type");
            }
            t.cols.push_back(std::move(col));
        }
        computeZones(t);
        *out = h;
        return VEXQ_OK;
    });
}

void ref_table_free(ref_table_t t) { delete t; }

int32_t ref_table_zone_map(ref_table_t t, int32_t col, int32_t rg, vexq_zone_map* out) {
    if (!t || col < 0 || col >= (int)t->t.cols.size() || rg < 0 || rg >= t->t.n_rg) return VEXQ_EINVAL;
    *out = t->t.cols[col].zones[rg];
    return VEXQ_OK;
}

int32_t ref_agg_run(ref_table_t t, const vexq_agg_plan_desc* d, int32_t rg_start, int32_t rg_end, int32_t workers,
                    ref_result_t* out) {
    return guarded([&]() -> int32_t {
        int rge = rg_end < 0 ? t->t.n_rg : std::min(rg_end, t->t.n_rg);
        *out = runAgg(t->t, d, std::max(0, rg_start), rge, workers);
        return VEXQ_OK;
    });
}

int32_t ref_join_run(ref_table_t build, ref_table_t probe, const vexq_join_plan_desc* d, int32_t workers,
                     ref_result_t* out) {
    return guarded([&]() -> int32_t {
        *out = runJoin(build->t, probe->t, d, workers);
        return VEXQ_OK;
    });
}

int32_t ref_zone_prune(ref_table_t t, const vexq_agg_plan_desc* d, uint8_t* mask, int32_t n_rg) {
    return guarded([&]() -> int32_t {
        Nodes N{d->nodes, d->nnodes, d->children, d->nchildren};
        for (int rg = 0; rg < n_rg && rg < t->t.n_rg; rg++)
            mask[rg] = d->predicate < 0 ? 1 : zoneEval(N, d->predicate, t->t, rg);
        return VEXQ_OK;
    });
}

int32_t ref_filter_run(ref_table_t t, const vexq_expr* nodes, int32_t nnodes, const int32_t* children,
                       int32_t nchildren, int32_t predicate, uint8_t* out_bits, int64_t* count) {
    return guarded([&]() -> int32_t {
        Nodes N{nodes, nnodes, children, nchildren};
        Schema s = tableSchema(t->t);
        XP pred = build(N, predicate, s);
        if (pred->type != VEXQ_TYPE_BOOL) throw Error("filter predicate must return BOOL");
        const Table& tb = t->t;
        std::memset(out_bits, 0, (size_t)((tb.nrows + 7) / 8));
        int64_t cnt = 0;
        Scan sc(&tb);
        Batch b;
        for (int rg = 0; rg < tb.n_rg; rg++) {
            for (int64_t s0 = tb.rgStart(rg); s0 < tb.rgEnd(rg); s0 += kBlockRows) {
                int n = (int)std::min<int64_t>(kBlockRows, tb.rgEnd(rg) - s0);
                sc.load(rg, s0, n, b);
                selectInto(b, eval(pred.get(), b));
                for (uint16_t i : b.sel) {
                    int64_t r = s0 + i;
                    out_bits[r >> 3] |= (uint8_t)(1u << (r & 7));
                    cnt++;
                }
            }
        }
        *count = cnt;
        return VEXQ_OK;
    });
}

// TableScan (zone-map skip, exec/scan.go:212-215) → Filter (filter.go:49-78,
// BoolToSelVecInto) → Project (project.go:64-128): each expression evaluated
// over the batch's physical rows and materialised through the SelVec
// (Project.materialize), batches concatenated in row order. The zone check
// uses the predicate tree, as planner.Physical hands TableScan its zonePred.
int32_t ref_project_run(ref_table_t t, const vexq_expr* nodes, int32_t nnodes, const int32_t* children,
                        int32_t nchildren, int32_t predicate, const int32_t* roots, int32_t nroots, int32_t rg_start,
                        int32_t rg_end, ref_result_t* out) {
    return guarded([&]() -> int32_t {
        Nodes N{nodes, nnodes, children, nchildren};
        const Table& tb = t->t;
        Schema s = tableSchema(tb);
        XP pred;
        if (predicate >= 0) {
            pred = build(N, predicate, s);
            if (pred->type != VEXQ_TYPE_BOOL) throw Error("filter predicate must return BOOL");
        }
        std::vector<XP> ex;
        for (int j = 0; j < nroots; j++) ex.push_back(build(N, roots[j], s));
        auto* r = new ref_result_s;
        std::unique_ptr<ref_result_s> keep(r);
        r->cols.resize(nroots);
        for (int j = 0; j < nroots; j++) r->cols[j].type = ex[j]->type;
        const int rge = rg_end < 0 ? tb.n_rg : std::min(rg_end, tb.n_rg);
        Scan sc(&tb);
        Batch b;
        Vec m;
        for (int rg = std::max(0, rg_start); rg < rge; rg++) {
            if (predicate >= 0 && !zoneEval(N, predicate, tb, rg)) continue;
            for (int64_t s0 = tb.rgStart(rg); s0 < tb.rgEnd(rg); s0 += kBlockRows) {
                const int n = (int)std::min<int64_t>(kBlockRows, tb.rgEnd(rg) - s0);
                sc.load(rg, s0, n, b);
                if (pred) {
                    selectInto(b, eval(pred.get(), b));
                    if (b.sel.empty()) continue;
                }
                for (int j = 0; j < nroots; j++) {
                    const Vec* v = eval(ex[j].get(), b);
                    const Vec* src = v;
                    if (b.has_sel) { materialize(*v, b.sel, m); src = &m; }
                    OutCol& oc = r->cols[j];
                    for (int i = 0; i < src->n; i++) {
                        oc.bits.push_back(src->valid[i] ? extractInt64(*src, i) : 0);
                        oc.valid.push_back(src->valid[i]);
                        oc.strs.push_back(src->type == VEXQ_TYPE_STRING && src->valid[i] ? src->str(i) : std::string());
                        oc.exact.push_back(std::nan(""));
                    }
                }
                r->rows += b.rows();
            }
        }
        *out = keep.release();
        return VEXQ_OK;
    });
}

// HAVING (planner/build.go:59-75): the Filter above the aggregate runs over
// the aggregate's output batches with the WHERE machinery, so the output
// columns become a one-row-group table scanned and filtered like any other;
// then buildHavingProjection keeps the first `visible` columns
// (planner/build.go:617-637) and ExternalSort + Limit run on what is left.
int32_t ref_result_having(ref_result_t r, const vexq_expr* nodes, int32_t nnodes, const int32_t* children,
                          int32_t nchildren, int32_t predicate, int32_t visible, const vexq_order_desc* order) {
    return guarded([&]() -> int32_t {
        const int64_t n = r->rows;
        Table t;
        t.nrows = n;
        t.rg_rows = (int)std::max<int64_t>(n, 1);
        t.n_rg = n > 0 ? 1 : 0;
        for (const OutCol& oc : r->cols) {
            Column col;
            col.name = oc.name;
            col.type = oc.type;
            col.nullable = true;
            col.valid = oc.valid;
            switch (oc.type) {
                case VEXQ_TYPE_INT64: col.i64 = oc.bits; break;
                case VEXQ_TYPE_FLOAT64:
                    col.f64.resize(n);
                    for (int64_t i = 0; i < n; i++) col.f64[i] = bitsToF(oc.bits[i]);
                    break;
                case VEXQ_TYPE_DATE:
                    col.i32.resize(n);
                    for (int64_t i = 0; i < n; i++) col.i32[i] = (int32_t)oc.bits[i];
                    break;
                case VEXQ_TYPE_BOOL:
                    col.b8.resize(n);
                    for (int64_t i = 0; i < n; i++) col.b8[i] = oc.bits[i] != 0;
                    break;
                case VEXQ_TYPE_STRING: {  // newStringVector: the batch's strings in first-occurrence order
                    auto dict = std::make_shared<Dict>();
                    col.codes.assign(n, 0);
                    for (int64_t i = 0; i < n; i++)
                        if (oc.valid[i]) col.codes[i] = dict->add(oc.strs[i]);
                    if (t.n_rg) col.dicts.push_back(dict);
                    break;
                }
                default: throw Error("unknown output column type");
            }
            t.cols.push_back(std::move(col));
        }
        computeZones(t);
        std::vector<int64_t> keep;
        if (predicate >= 0) {
            Nodes N{nodes, nnodes, children, nchildren};
            Schema sch = tableSchema(t);
            XP pred = build(N, predicate, sch);
            if (pred->type != VEXQ_TYPE_BOOL) throw Error("HAVING predicate must return BOOL");
            Scan sc(&t);
            Batch b;
            for (int64_t s0 = 0; s0 < n; s0 += kBlockRows) {
                const int m = (int)std::min<int64_t>(kBlockRows, n - s0);
                sc.load(0, s0, m, b);
                selectInto(b, eval(pred.get(), b));
                for (uint16_t i : b.sel) keep.push_back(s0 + i);
            }
        } else {
            for (int64_t i = 0; i < n; i++) keep.push_back(i);
        }
        for (auto& c : r->cols) {
            OutCol k = c;
            k.bits.resize(keep.size());
            k.valid.resize(keep.size());
            k.strs.resize(keep.size());
            k.exact.resize(keep.size());
            for (size_t j = 0; j < keep.size(); j++) {
                k.bits[j] = c.bits[keep[j]];
                k.valid[j] = c.valid[keep[j]];
                k.strs[j] = c.strs[keep[j]];
                k.exact[j] = c.exact[keep[j]];
            }
            c = std::move(k);
        }
        r->rows = (int64_t)keep.size();
        if (visible >= 0 && visible < (int)r->cols.size()) r->cols.resize(visible);
        if (order) applyOrder(r, *order);
        return VEXQ_OK;
    });
}

int64_t ref_result_rows(ref_result_t r) { return r ? r->rows : 0; }
int32_t ref_result_cols(ref_result_t r) { return r ? (int32_t)r->cols.size() : 0; }
int32_t ref_result_col_type(ref_result_t r, int32_t col) { return r->cols[col].type; }
const char* ref_result_col_name(ref_result_t r, int32_t col) { return r->cols[col].name.c_str(); }

int32_t ref_result_get(ref_result_t r, int64_t row, int32_t col, int64_t* bits, int32_t* valid, const char** str,
                       int32_t* len) {
    if (!r || col < 0 || col >= (int)r->cols.size() || row < 0 || row >= r->rows) return VEXQ_EINVAL;
    const OutCol& c = r->cols[col];
    *bits = c.bits[row];
    *valid = c.valid[row];
    *str = c.strs[row].data();
    *len = (int32_t)c.strs[row].size();
    return VEXQ_OK;
}

int32_t ref_result_exact(ref_result_t r, int64_t row, int32_t col, double* out) {
    if (!r || col < 0 || col >= (int)r->cols.size() || row < 0 || row >= r->rows) return VEXQ_EINVAL;
    *out = r->cols[col].exact[row];
    return VEXQ_OK;
}

void ref_result_free(ref_result_t r) { delete r; }

}  // extern "C"
