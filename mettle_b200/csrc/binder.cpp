// binder.cpp — AST -> typed BoundPlan.
//
// Resolves tables against the pinned catalog, splits WHERE into per-table
// predicates and equi-join edges (the reference's parse_where_clause,
// src/plan/parser.rs:244-343, and its join-constraint extraction,
// parser.rs:138-210), and types every expression with DuckDB's rules so
// integer, DECIMAL and date results are exact: the reference evaluates all
// expressions in f32 on the GPU (src/plan/helpers.rs:141-206) and in f64 on
// the CPU (helpers.rs:234-328).
#include <cmath>
#include <cstring>
#include <algorithm>

#include "engine.h"

namespace mtl {

namespace {

using i128 = __int128;

const i128 kI64Max = (i128)INT64_MAX;
const i128 kI64Min = (i128)INT64_MIN;

int64_t pow10i(int n) {
  int64_t r = 1;
  for (int i = 0; i < n; ++i) r *= 10;
  return r;
}
i128 pow10w(int n) {
  i128 r = 1;
  for (int i = 0; i < n; ++i) r *= 10;
  return r;
}

int digits_of(i128 v) {
  if (v < 0) v = -v;
  int d = 1;
  while (v >= 10) {
    v /= 10;
    ++d;
  }
  return d;
}

LType T(int t, int w = 0, int s = 0) {
  LType x;
  x.t = t;
  x.width = w;
  x.scale = s;
  return x;
}

struct Binder {
  Ctx& ctx;
  BoundPlan& plan;

  // ------------------------------------------------------------ sources
  int find_source(const std::string& qual) const {
    for (size_t i = 0; i < plan.sources.size(); ++i) {
      const Source& s = plan.sources[i];
      if (!s.alias.empty() ? s.alias == qual : s.name == qual) return (int)i;
    }
    for (size_t i = 0; i < plan.sources.size(); ++i)
      if (plan.sources[i].name == qual) return (int)i;
    return -1;
  }

  std::pair<int, Column*> resolve(const Ast& a) const {
    if (!a.table.empty()) {
      int s = find_source(a.table);
      if (s < 0) fail(MTL_INVALID, "referenced table \"" + a.table + "\" not found in FROM clause");
      Column* c = plan.sources[s].table->find(a.name);
      if (!c) fail(MTL_INVALID, "column \"" + a.name + "\" not found in table \"" + a.table + "\"");
      return {s, c};
    }
    int found = -1;
    Column* fc = nullptr;
    for (size_t i = 0; i < plan.sources.size(); ++i) {
      Column* c = plan.sources[i].table->find(a.name);
      if (c) {
        if (found >= 0) fail(MTL_INVALID, "ambiguous reference to column name \"" + a.name + "\"");
        found = (int)i;
        fc = c;
      }
    }
    if (found < 0) fail(MTL_INVALID, "referenced column \"" + a.name + "\" not found");
    return {found, fc};
  }

  // ------------------------------------------------------------ literals
  BExprP make_const(LType t, int32_t ptype, int64_t lo, int64_t hi = 0) {
    auto e = std::make_shared<BExpr>();
    e->k = BExpr::CONST;
    e->type = t;
    e->ptype = ptype;
    e->lo = lo;
    e->hi = hi;
    if (ptype == P_I32 || ptype == P_I64 || ptype == P_I128) {
      i128 v = ptype == P_I128 ? (i128)(((unsigned __int128)(uint64_t)hi << 64) | (uint64_t)lo) : (i128)lo;
      e->bounded = true;
      e->bmin = e->bmax = v;
    }
    return e;
  }

  static double const_as_double(const BExpr& c) {
    switch (c.ptype) {
      case P_F32: {
        float f;
        uint32_t b = (uint32_t)c.lo;
        memcpy(&f, &b, 4);
        return f;
      }
      case P_F64: {
        double d;
        memcpy(&d, &c.lo, 8);
        return d;
      }
      case P_I128: return (double)(i128)(((unsigned __int128)(uint64_t)c.hi << 64) | (uint64_t)c.lo);
      default: return (double)c.lo;
    }
  }

  // Parses a decimal literal "123.456" exactly into (value, width, scale).
  static bool parse_decimal(const std::string& s, i128* v, int* w, int* sc) {
    i128 x = 0;
    int scale = 0, digits = 0;
    bool dot = false;
    for (char c : s) {
      if (c == '.') {
        if (dot) return false;
        dot = true;
        continue;
      }
      if (c < '0' || c > '9') return false;
      x = x * 10 + (c - '0');
      if (x != 0 || dot) ++digits;
      if (dot) ++scale;
      if (digits > 38) return false;
    }
    *v = x;
    *sc = scale;
    *w = std::max(digits, scale) > 0 ? std::max(std::max(digits, scale), 1) : 1;
    if (*w < *sc) *w = *sc;
    return true;
  }

  // ------------------------------------------------------------ casts
  // Casts e (non-constant) to logical type `to` with VM representation pt.
  BExprP cast_to(BExprP e, LType to, int32_t pt) {
    if (e->k == BExpr::CONST) return cast_const(*e, to, pt);
    int64_t mul = 1, div = 1;
    if (is_decimal(to) && (is_decimal(e->type) || is_int_family(e->type))) {
      int from_s = is_decimal(e->type) ? e->type.scale : 0;
      if (to.scale < from_s) fail(MTL_UNSUPPORTED, "decimal down-scaling is not supported");
      mul = pow10i(to.scale - from_s);
    }
    if (is_float_family(to) && is_decimal(e->type)) div = pow10i(e->type.scale);
    if (e->ptype == pt && mul == 1 && div == 1) {
      if (e->type.t == to.t && e->type.scale == to.scale) return e;
      auto c = std::make_shared<BExpr>(*e);
      c->type = to;
      return c;
    }
    auto c = std::make_shared<BExpr>();
    c->k = BExpr::CAST;
    c->type = to;
    c->ptype = pt;
    c->mul = mul;
    c->div = div;
    c->a = {e};
    c->text = e->text;
    if (e->bounded && (pt == P_I32 || pt == P_I64 || pt == P_I128)) {
      c->bounded = true;
      c->bmin = e->bmin * (i128)mul;
      c->bmax = e->bmax * (i128)mul;
    }
    return c;
  }

  BExprP cast_const(const BExpr& c, LType to, int32_t pt) {
    if (pt == P_F32 || pt == P_F64) {
      double d;
      if (c.ptype == P_F32 || c.ptype == P_F64) {
        d = const_as_double(c);
      } else {
        i128 v = c.ptype == P_I128 ? (i128)(((unsigned __int128)(uint64_t)c.hi << 64) | (uint64_t)c.lo) : (i128)c.lo;
        if (is_decimal(c.type) && c.type.scale > 0) {
          // DuckDB decimal -> float: integer value / 10^scale in the target type.
          if (pt == P_F32) {
            float f = (float)(double)v / (float)pow10i(c.type.scale);
            return make_const(to, pt, (int64_t)(uint32_t)*(uint32_t*)&f);
          }
          d = (double)v / (double)pow10i(c.type.scale);
        } else {
          if (pt == P_F32) {
            float f = (float)v;
            return make_const(to, pt, (int64_t)(uint32_t)*(uint32_t*)&f);
          }
          d = (double)v;
        }
      }
      if (pt == P_F32) {
        float f = (float)d;
        uint32_t b;
        memcpy(&b, &f, 4);
        return make_const(to, pt, (int64_t)b);
      }
      int64_t b;
      memcpy(&b, &d, 8);
      return make_const(to, pt, b);
    }
    if (c.ptype == P_F32 || c.ptype == P_F64) fail(MTL_UNSUPPORTED, "float to integer cast is not supported");
    i128 v = c.ptype == P_I128 ? (i128)(((unsigned __int128)(uint64_t)c.hi << 64) | (uint64_t)c.lo) : (i128)c.lo;
    int from_s = is_decimal(c.type) ? c.type.scale : 0;
    int to_s = is_decimal(to) ? to.scale : 0;
    if (to_s < from_s) fail(MTL_UNSUPPORTED, "decimal down-scaling is not supported");
    v *= pow10w(to_s - from_s);
    if (pt == P_I32 && (v > INT32_MAX || v < INT32_MIN)) fail(MTL_OVERFLOW, "Overflow in cast of constant");
    if (pt == P_I64 && (v > kI64Max || v < kI64Min)) fail(MTL_OVERFLOW, "Overflow in cast of constant");
    auto e = make_const(to, pt, (int64_t)(uint64_t)v, (int64_t)(v >> 64));
    e->is_int_literal = c.is_int_literal;
    return e;
  }

  // ------------------------------------------------------------ bounds
  void col_bounds(BExpr& e) {
    Column& c = *e.col;
    if (!(c.type.t == MTL_T_INTEGER || c.type.t == MTL_T_BIGINT || c.type.t == MTL_T_DECIMAL ||
          c.type.t == MTL_T_DATE || c.type.t == MTL_T_TIMESTAMP))
      return;
    column_minmax(ctx, c);
    if (c.has_minmax) {
      e.bounded = true;
      e.bmin = c.vmin;
      e.bmax = c.vmax;
    }
  }

  static void arith_bounds(BExpr& r, const BExpr& a, const BExpr& b) {
    if (!a.bounded || !b.bounded) return;
    const i128 lim = ((i128)1) << 100;
    auto ok = [&](i128 x) { return x < lim && x > -lim; };
    if (!ok(a.bmin) || !ok(a.bmax) || !ok(b.bmin) || !ok(b.bmax)) return;
    i128 c[4];
    switch (r.op) {
      case VM_ADD: r.bmin = a.bmin + b.bmin; r.bmax = a.bmax + b.bmax; break;
      case VM_SUB: r.bmin = a.bmin - b.bmax; r.bmax = a.bmax - b.bmin; break;
      default: {
        const i128 l2 = ((i128)1) << 62;
        if (!(a.bmin > -l2 && a.bmax < l2 && b.bmin > -l2 && b.bmax < l2)) return;
        c[0] = a.bmin * b.bmin; c[1] = a.bmin * b.bmax; c[2] = a.bmax * b.bmin; c[3] = a.bmax * b.bmax;
        r.bmin = *std::min_element(c, c + 4);
        r.bmax = *std::max_element(c, c + 4);
      }
    }
    r.bounded = true;
  }

  static bool fits64(const BExpr& e) { return e.bounded && e.bmin >= kI64Min && e.bmax <= kI64Max; }

  // ------------------------------------------------------------ expressions
  BExprP bind_expr(const AstP& a) {
    switch (a->k) {
      case Ast::COL: {
        auto [s, c] = resolve(*a);
        auto e = std::make_shared<BExpr>();
        e->k = BExpr::COL;
        e->src = s;
        e->col = c;
        e->type = c->type;
        e->ptype = storage_ptype(c->type);
        e->text = a->name;
        col_bounds(*e);
        return e;
      }
      case Ast::INT: {
        errno = 0;
        char* end = nullptr;
        long long v = strtoll(a->name.c_str(), &end, 10);
        if (errno == ERANGE || *end) {
          i128 x;
          int w, sc;
          if (!parse_decimal(a->name, &x, &w, &sc)) fail(MTL_INVALID, "bad integer literal");
          auto e = make_const(T(MTL_T_HUGEINT), P_I128, (int64_t)(uint64_t)x, (int64_t)(x >> 64));
          e->is_int_literal = true;
          e->text = a->text;
          return e;
        }
        LType t = (v >= INT32_MIN && v <= INT32_MAX) ? T(MTL_T_INTEGER) : T(MTL_T_BIGINT);
        auto e = make_const(t, t.t == MTL_T_INTEGER ? P_I32 : P_I64, v);
        e->is_int_literal = true;
        e->text = a->text;
        return e;
      }
      case Ast::DEC: {
        if (a->name.find_first_of("eE") != std::string::npos) {
          double d = strtod(a->name.c_str(), nullptr);
          int64_t b;
          memcpy(&b, &d, 8);
          auto e = make_const(T(MTL_T_DOUBLE), P_F64, b);
          e->text = a->text;
          return e;
        }
        i128 v;
        int w, sc;
        if (!parse_decimal(a->name, &v, &w, &sc)) fail(MTL_INVALID, "bad decimal literal");
        LType t = T(MTL_T_DECIMAL, w, sc);
        int32_t pt = w <= 18 ? P_I64 : P_I128;
        if (w > 18) t.t = MTL_T_DECIMAL128;
        auto e = make_const(t, pt, (int64_t)(uint64_t)v, (int64_t)(v >> 64));
        e->is_dec_literal = true;
        e->text = a->text;
        return e;
      }
      case Ast::DATE: {
        int32_t d;
        if (!parse_date(a->name, &d)) fail(MTL_INVALID, "invalid date literal '" + a->name + "'");
        auto e = make_const(T(MTL_T_DATE), P_I32, d);
        e->text = a->text;
        return e;
      }
      case Ast::TS: {
        int64_t us;
        if (!parse_timestamp(a->name, &us)) fail(MTL_INVALID, "invalid timestamp literal '" + a->name + "'");
        auto e = make_const(T(MTL_T_TIMESTAMP), P_I64, us);
        e->text = a->text;
        return e;
      }
      case Ast::NEG: {
        BExprP x = bind_expr(a->a[0]);
        if (x->k == BExpr::CONST) {
          if (x->ptype == P_F32) x->lo ^= 0x80000000LL;
          else if (x->ptype == P_F64) x->lo ^= (int64_t)0x8000000000000000ULL;
          else {
            i128 v = x->ptype == P_I128 ? (i128)(((unsigned __int128)(uint64_t)x->hi << 64) | (uint64_t)x->lo)
                                       : (i128)x->lo;
            v = -v;
            x->lo = (int64_t)(uint64_t)v;
            x->hi = (int64_t)(v >> 64);
            x->bmin = x->bmax = v;
          }
          x->text = a->text;
          return x;
        }
        if (x->type.t == MTL_T_VARCHAR || x->type.t == MTL_T_DATE || x->type.t == MTL_T_TIMESTAMP)
          fail(MTL_INVALID, "cannot negate " + type_name(x->type));
        auto e = std::make_shared<BExpr>();
        e->k = BExpr::NEG;
        e->type = x->type;
        e->ptype = x->ptype;
        e->a = {x};
        e->text = a->text;
        if (x->bounded) {
          e->bounded = true;
          e->bmin = -x->bmax;
          e->bmax = -x->bmin;
        }
        return e;
      }
      case Ast::BIN: {
        if (a->op == '/' || a->op == '%' || a->op == '|')
          fail(MTL_UNSUPPORTED, std::string("operator '") + a->op + "' is outside the offloaded subset");
        BExprP l = bind_expr(a->a[0]);
        BExprP r = bind_expr(a->a[1]);
        BExprP e = bind_arith(a->op == '+' ? VM_ADD : a->op == '-' ? VM_SUB : VM_MUL, l, r);
        e->text = a->text;
        return e;
      }
      case Ast::STR:
        fail(MTL_UNSUPPORTED, "string expressions are outside the offloaded subset");
      case Ast::FUNC:
        fail(MTL_UNSUPPORTED, "function " + a->name + "() is outside the offloaded subset here");
      default:
        fail(MTL_UNSUPPORTED, "expression '" + a->text + "' is outside the offloaded subset");
    }
  }

  static int int_rank(int t) { return t == MTL_T_INTEGER ? 1 : t == MTL_T_BIGINT ? 2 : 3; }
  static int32_t int_ptype(int t) { return t == MTL_T_INTEGER ? P_I32 : t == MTL_T_BIGINT ? P_I64 : P_I128; }

  // Decimal image of an integer-family operand: DECIMAL(w, 0).
  static LType dec_of_int(const BExpr& e) {
    if (e.k == BExpr::CONST) {
      i128 v = e.ptype == P_I128 ? (i128)(((unsigned __int128)(uint64_t)e.hi << 64) | (uint64_t)e.lo) : (i128)e.lo;
      return T(MTL_T_DECIMAL, digits_of(v), 0);
    }
    return T(MTL_T_DECIMAL, e.type.t == MTL_T_INTEGER ? 10 : e.type.t == MTL_T_BIGINT ? 19 : 38, 0);
  }

  BExprP fold(int16_t op, const BExpr& l, const BExpr& r, LType t, int32_t pt) {
    if (pt == P_F32 || pt == P_F64) {
      double x = const_as_double(l), y = const_as_double(r);
      if (pt == P_F32) {
        float fx = (float)x, fy = (float)y;
        volatile float v = op == VM_ADD ? fx + fy : op == VM_SUB ? fx - fy : fx * fy;
        float vv = v;
        uint32_t b;
        memcpy(&b, &vv, 4);
        return make_const(t, pt, (int64_t)b);
      }
      volatile double v = op == VM_ADD ? x + y : op == VM_SUB ? x - y : x * y;
      double vv = v;
      int64_t b;
      memcpy(&b, &vv, 8);
      return make_const(t, pt, b);
    }
    auto iv = [](const BExpr& c) {
      return c.ptype == P_I128 ? (i128)(((unsigned __int128)(uint64_t)c.hi << 64) | (uint64_t)c.lo) : (i128)c.lo;
    };
    i128 x = iv(l), y = iv(r);
    i128 v = op == VM_ADD ? x + y : op == VM_SUB ? x - y : x * y;
    if (pt == P_I32 && (v > INT32_MAX || v < INT32_MIN)) fail(MTL_OVERFLOW, "Overflow in constant arithmetic");
    if (pt == P_I64 && (v > kI64Max || v < kI64Min)) fail(MTL_OVERFLOW, "Overflow in constant arithmetic");
    return make_const(t, pt, (int64_t)(uint64_t)v, (int64_t)(v >> 64));
  }

  BExprP bind_arith(int16_t op, BExprP l, BExprP r) {
    const LType lt = l->type, rt = r->type;
    if (lt.t == MTL_T_VARCHAR || rt.t == MTL_T_VARCHAR) fail(MTL_INVALID, "arithmetic on VARCHAR");
    if (lt.t == MTL_T_TIMESTAMP || rt.t == MTL_T_TIMESTAMP)
      fail(MTL_UNSUPPORTED, "TIMESTAMP arithmetic is outside the offloaded subset");
    LType res;
    int32_t pt;
    if (lt.t == MTL_T_DATE || rt.t == MTL_T_DATE) {
      // DATE +/- INTEGER -> DATE (days).
      bool ok = (lt.t == MTL_T_DATE && is_int_family(rt) && op != VM_MUL) ||
                (rt.t == MTL_T_DATE && is_int_family(lt) && op == VM_ADD);
      if (!ok) fail(MTL_UNSUPPORTED, "date arithmetic other than DATE +/- INTEGER");
      res = T(MTL_T_DATE);
      pt = P_I32;
      l = cast_to(l, lt.t == MTL_T_DATE ? lt : T(MTL_T_INTEGER), P_I32);
      r = cast_to(r, rt.t == MTL_T_DATE ? rt : T(MTL_T_INTEGER), P_I32);
    } else if (lt.t == MTL_T_DOUBLE || rt.t == MTL_T_DOUBLE) {
      res = T(MTL_T_DOUBLE);
      pt = P_F64;
      l = cast_to(l, res, pt);
      r = cast_to(r, res, pt);
    } else if (lt.t == MTL_T_FLOAT || rt.t == MTL_T_FLOAT) {
      res = T(MTL_T_FLOAT);
      pt = P_F32;
      l = cast_to(l, res, pt);
      r = cast_to(r, res, pt);
    } else if (is_decimal(lt) || is_decimal(rt)) {
      LType dl = is_decimal(lt) ? lt : dec_of_int(*l);
      LType dr = is_decimal(rt) ? rt : dec_of_int(*r);
      int s, w;
      if (op == VM_MUL) {
        s = dl.scale + dr.scale;
        w = std::min(38, dl.width + dr.width);
      } else {
        s = std::max(dl.scale, dr.scale);
        w = std::min(38, std::max(dl.width - dl.scale, dr.width - dr.scale) + s + 1);
      }
      res = T(w <= 18 ? MTL_T_DECIMAL : MTL_T_DECIMAL128, w, s);
      // operands at their own scale (MUL) or the common scale (ADD/SUB)
      LType tl = T(dl.width <= 18 ? MTL_T_DECIMAL : MTL_T_DECIMAL128, dl.width, op == VM_MUL ? dl.scale : s);
      LType tr = T(dr.width <= 18 ? MTL_T_DECIMAL : MTL_T_DECIMAL128, dr.width, op == VM_MUL ? dr.scale : s);
      // Work in I64 when the value ranges allow it, else I128.
      int32_t ptl = P_I128, ptr = P_I128;
      BExprP cl = cast_to(l, tl, P_I128), cr = cast_to(r, tr, P_I128);
      if (fits64(*cl)) ptl = P_I64;
      if (fits64(*cr)) ptr = P_I64;
      BExpr tmp;
      tmp.op = op;
      arith_bounds(tmp, *cl, *cr);
      pt = (ptl == P_I64 && ptr == P_I64 && fits64(tmp)) ? P_I64 : P_I128;
      l = cast_to(l, tl, pt);
      r = cast_to(r, tr, pt);
    } else {
      // integer family; a literal adopts the column's type when it fits
      int rank = std::max(int_rank(lt.t), int_rank(rt.t));
      if (l->is_int_literal && !r->is_int_literal && r->k != BExpr::CONST) rank = std::max(int_rank(rt.t), rank == 3 ? 3 : int_rank(rt.t));
      if (r->is_int_literal && !l->is_int_literal && l->k != BExpr::CONST) rank = std::max(int_rank(lt.t), rank == 3 ? 3 : int_rank(lt.t));
      if (l->is_int_literal && int_rank(l->type.t) > rank) rank = int_rank(l->type.t);
      if (r->is_int_literal && int_rank(r->type.t) > rank) rank = int_rank(r->type.t);
      res = T(rank == 1 ? MTL_T_INTEGER : rank == 2 ? MTL_T_BIGINT : MTL_T_HUGEINT);
      pt = int_ptype(res.t);
      l = cast_to(l, res, pt);
      r = cast_to(r, res, pt);
    }
    if (l->k == BExpr::CONST && r->k == BExpr::CONST) return fold(op, *l, *r, res, pt);
    auto e = std::make_shared<BExpr>();
    e->k = BExpr::ARITH;
    e->op = op;
    e->type = res;
    e->ptype = pt;
    e->a = {l, r};
    arith_bounds(*e, *l, *r);
    return e;
  }

  // ------------------------------------------------------------ predicates
  void add_filter(int src, Column* c, int op, const BExprP& lit) {
    BFilter f;
    f.src = src;
    f.col = c;
    const LType& ct = c->type;
    const BExpr& L = *lit;
    auto ival = [&](const BExpr& x) {
      return x.ptype == P_I128 ? (i128)(((unsigned __int128)(uint64_t)x.hi << 64) | (uint64_t)x.lo) : (i128)x.lo;
    };
    // Integer-domain compare of column value x (scaled by 10^cs) against a
    // literal v / 10^ls: exact rewrite to an integer bound.
    auto int_pred = [&](i128 num, i128 den) {
      // predicate: x op num/den, den > 0
      auto floor_div = [](i128 a, i128 b) {
        i128 q = a / b;
        if ((a % b != 0) && ((a < 0) != (b < 0))) --q;
        return q;
      };
      i128 fl = floor_div(num, den);
      bool exact = (num % den) == 0;
      i128 ce = exact ? fl : fl + 1;
      switch (op) {
        case C_EQ:
          if (!exact) f.op = C_FALSE;
          else { f.op = C_EQ; f.ilit = (int64_t)fl; }
          break;
        case C_NE:
          if (!exact) f.op = C_TRUE;
          else { f.op = C_NE; f.ilit = (int64_t)fl; }
          break;
        case C_LT: f.op = exact ? C_LT : C_LE; f.ilit = (int64_t)(exact ? fl : fl); break;
        case C_LE: f.op = C_LE; f.ilit = (int64_t)fl; break;
        case C_GT: f.op = C_GE; f.ilit = (int64_t)(exact ? fl + 1 : ce); break;
        case C_GE: f.op = C_GE; f.ilit = (int64_t)ce; break;
      }
      if (fl > kI64Max || fl < kI64Min) {
        // literal outside the column's range: decide statically
        bool above = num > 0;
        bool r = (op == C_LT || op == C_LE) ? above : (op == C_GT || op == C_GE) ? !above : op == C_NE;
        f.op = r ? C_TRUE : C_FALSE;
      }
    };
    switch (ct.t) {
      case MTL_T_INTEGER:
      case MTL_T_BIGINT:
      case MTL_T_DECIMAL: {
        int cs = ct.t == MTL_T_DECIMAL ? ct.scale : 0;
        if (L.ptype == P_F32 || L.ptype == P_F64) {
          double d = const_as_double(L) * std::pow(10.0, cs);
          double fl = std::floor(d);
          i128 num = (i128)fl;
          if (fl == d) int_pred(num, 1);
          else int_pred(num * 2 + 1, 2);  // strictly between fl and fl+1
        } else if (is_int_family(L.type) || is_decimal(L.type)) {
          int ls = is_decimal(L.type) ? L.type.scale : 0;
          i128 v = ival(L);
          if (ls <= cs) int_pred(v * pow10w(cs - ls), 1);
          else int_pred(v, pow10w(ls - cs));
        } else {
          fail(MTL_INVALID, "cannot compare " + type_name(ct) + " with " + type_name(L.type));
        }
        break;
      }
      case MTL_T_DATE:
        if (L.type.t == MTL_T_DATE) {
          f.op = op;
          f.ilit = L.lo;
        } else if (L.type.t == MTL_T_TIMESTAMP) {
          // DATE column vs TIMESTAMP literal compares as timestamps.
          int64_t us = L.lo, day = 86400000000LL;
          i128 num = us, den = day;
          int_pred(num, den);
        } else {
          fail(MTL_INVALID, "cannot compare DATE with " + type_name(L.type));
        }
        break;
      case MTL_T_TIMESTAMP:
        if (L.type.t == MTL_T_TIMESTAMP) {
          f.op = op;
          f.ilit = L.lo;
        } else if (L.type.t == MTL_T_DATE) {
          f.op = op;
          f.ilit = L.lo * 86400000000LL;
        } else {
          fail(MTL_INVALID, "cannot compare TIMESTAMP with " + type_name(L.type));
        }
        break;
      case MTL_T_FLOAT:
      case MTL_T_DOUBLE:
        if (L.type.t == MTL_T_VARCHAR || L.type.t == MTL_T_DATE || L.type.t == MTL_T_TIMESTAMP)
          fail(MTL_INVALID, "cannot compare " + type_name(ct) + " with " + type_name(L.type));
        f.op = op;
        if (ct.t == MTL_T_FLOAT) {
          // the literal is cast to FLOAT, then compared in binary32
          BExprP fc = cast_const(L, T(MTL_T_FLOAT), P_F32);
          f.flit = const_as_double(*fc);
        } else {
          BExprP dc = cast_const(L, T(MTL_T_DOUBLE), P_F64);
          f.flit = const_as_double(*dc);
        }
        break;
      default:
        fail(MTL_INVALID, "unsupported comparison on " + type_name(ct));
    }
    plan.filters.push_back(f);
  }

  void add_string_filter(int src, Column* c, int op, const std::string& s) {
    if (c->type.t == MTL_T_DATE || c->type.t == MTL_T_TIMESTAMP) {
      BExprP lit;
      if (c->type.t == MTL_T_DATE) {
        int32_t d;
        if (!parse_date(s, &d)) fail(MTL_INVALID, "invalid date '" + s + "'");
        lit = make_const(T(MTL_T_DATE), P_I32, d);
      } else {
        int64_t us;
        if (!parse_timestamp(s, &us)) fail(MTL_INVALID, "invalid timestamp '" + s + "'");
        lit = make_const(T(MTL_T_TIMESTAMP), P_I64, us);
      }
      add_filter(src, c, op, lit);
      return;
    }
    if (c->type.t != MTL_T_VARCHAR) fail(MTL_INVALID, "cannot compare " + type_name(c->type) + " with VARCHAR");
    BFilter f;
    f.src = src;
    f.col = c;
    const auto& d = c->dict;
    int64_t lb = std::lower_bound(d.begin(), d.end(), s) - d.begin();
    int64_t ub = std::upper_bound(d.begin(), d.end(), s) - d.begin();
    bool present = lb < ub;
    switch (op) {
      case C_EQ: f.op = present ? C_EQ : C_FALSE; f.ilit = lb; break;
      case C_NE: f.op = present ? C_NE : C_TRUE; f.ilit = lb; break;
      case C_LT: f.op = C_LT; f.ilit = lb; break;
      case C_LE: f.op = C_LT; f.ilit = ub; break;
      case C_GT: f.op = C_GE; f.ilit = ub; break;
      case C_GE: f.op = C_GE; f.ilit = lb; break;
      default: f.op = C_FALSE;
    }
    plan.filters.push_back(f);
  }

  static int flip(int op) {
    switch (op) {
      case C_LT: return C_GT;
      case C_LE: return C_GE;
      case C_GT: return C_LT;
      case C_GE: return C_LE;
      default: return op;
    }
  }

  bool is_literal_ast(const AstP& a) {
    if (a->k == Ast::INT || a->k == Ast::DEC || a->k == Ast::STR || a->k == Ast::DATE || a->k == Ast::TS) return true;
    if (a->k == Ast::NEG) return is_literal_ast(a->a[0]);
    if (a->k == Ast::BIN) return is_literal_ast(a->a[0]) && is_literal_ast(a->a[1]);
    return false;
  }

  void conjunct(const AstP& a) {
    switch (a->k) {
      case Ast::AND:
        conjunct(a->a[0]);
        conjunct(a->a[1]);
        return;
      case Ast::CMP: {
        const AstP& l = a->a[0];
        const AstP& r = a->a[1];
        if (l->k == Ast::COL && r->k == Ast::COL) {
          auto [ls, lc] = resolve(*l);
          auto [rs, rc] = resolve(*r);
          if (ls != rs && a->cmp == C_EQ) {
            BJoin j;
            j.ls = ls;
            j.lc = lc;
            j.rs = rs;
            j.rc = rc;
            plan.joins.push_back(j);
            return;
          }
          fail(MTL_UNSUPPORTED, "column-to-column predicate '" + a->text + "' is outside the offloaded subset");
        }
        const AstP* colp = nullptr;
        const AstP* litp = nullptr;
        int op = a->cmp;
        if (l->k == Ast::COL && is_literal_ast(r)) {
          colp = &l;
          litp = &r;
        } else if (r->k == Ast::COL && is_literal_ast(l)) {
          colp = &r;
          litp = &l;
          op = flip(op);
        } else {
          fail(MTL_UNSUPPORTED, "predicate '" + a->text + "' is outside the offloaded subset");
        }
        auto [s, c] = resolve(**colp);
        if ((*litp)->k == Ast::STR) {
          add_string_filter(s, c, op, (*litp)->name);
        } else {
          BExprP lit = bind_expr(*litp);
          if (lit->k != BExpr::CONST) fail(MTL_UNSUPPORTED, "non-constant predicate operand");
          add_filter(s, c, op, lit);
        }
        return;
      }
      case Ast::BETWEEN: {
        if (a->negated) fail(MTL_UNSUPPORTED, "NOT BETWEEN is outside the offloaded subset");
        // BETWEEN -> >= AND <= (src/plan/parser.rs:339-362)
        if (a->a[0]->k != Ast::COL) fail(MTL_UNSUPPORTED, "BETWEEN on an expression");
        auto [s, c] = resolve(*a->a[0]);
        for (int i = 1; i <= 2; ++i) {
          int op = i == 1 ? C_GE : C_LE;
          if (a->a[i]->k == Ast::STR) add_string_filter(s, c, op, a->a[i]->name);
          else {
            BExprP lit = bind_expr(a->a[i]);
            if (lit->k != BExpr::CONST) fail(MTL_UNSUPPORTED, "non-constant BETWEEN bound");
            add_filter(s, c, op, lit);
          }
        }
        return;
      }
      case Ast::OR:
        fail(MTL_UNSUPPORTED, "OR predicates are outside the offloaded subset");
      default:
        fail(MTL_UNSUPPORTED, "predicate '" + a->text + "' is outside the offloaded subset");
    }
  }

  // ------------------------------------------------------------ aggregates
  static bool is_agg_name(const std::string& n) {
    return n == "sum" || n == "count" || n == "min" || n == "max" || n == "avg" || n == "count_star";
  }
  static bool contains_agg(const AstP& a) {
    if (a->k == Ast::FUNC && is_agg_name(a->name)) return true;
    for (auto& c : a->a)
      if (contains_agg(c)) return true;
    return false;
  }

  int bind_agg(const AstP& a) {
    if (a->distinct) fail(MTL_UNSUPPORTED, "DISTINCT aggregates are outside the offloaded subset");
    BAgg g;
    g.text = a->text;
    const std::string& n = a->name;
    bool star = a->a.empty() || (a->a.size() == 1 && a->a[0]->k == Ast::STAR);
    if (n == "count" || n == "count_star") {
      g.fn = AG_COUNT;
      g.result = T(MTL_T_BIGINT);
      if (!star) {
        if (a->a.size() != 1) fail(MTL_INVALID, "count() takes one argument");
        g.arg = bind_expr(a->a[0]);  // no NULLs: COUNT(x) == COUNT(*)
        if (contains_agg(a->a[0])) fail(MTL_INVALID, "nested aggregates");
        g.arg = nullptr;
      }
    } else {
      if (star || a->a.size() != 1) fail(MTL_INVALID, n + "() takes one argument");
      if (contains_agg(a->a[0])) fail(MTL_INVALID, "nested aggregates");
      g.arg = bind_expr(a->a[0]);
      const LType at = g.arg->type;
      if (n == "sum") {
        g.fn = AG_SUM;
        if (is_int_family(at)) g.result = T(MTL_T_HUGEINT);
        else if (is_decimal(at)) g.result = T(MTL_T_DECIMAL128, 38, at.scale);
        else if (is_float_family(at)) g.result = T(MTL_T_DOUBLE);
        else fail(MTL_INVALID, "sum(" + type_name(at) + ") is not defined");
      } else if (n == "avg") {
        g.fn = AG_AVG;
        if (!(is_int_family(at) || is_decimal(at) || is_float_family(at)))
          fail(MTL_INVALID, "avg(" + type_name(at) + ") is not defined");
        g.result = T(MTL_T_DOUBLE);
      } else {
        g.fn = n == "min" ? AG_MIN : AG_MAX;
        if (at.t == MTL_T_DECIMAL128 || at.t == MTL_T_HUGEINT)
          fail(MTL_UNSUPPORTED, "min/max over 128-bit values");
        g.result = at;
      }
      if (g.arg->k == BExpr::COL) col_bounds(*g.arg);
    }
    // reuse an identical aggregate
    for (size_t i = 0; i < plan.aggs.size(); ++i)
      if (plan.aggs[i].fn == g.fn && plan.aggs[i].text == g.text) return (int)i;
    plan.aggs.push_back(g);
    return (int)plan.aggs.size() - 1;
  }

  static std::string agg_default_name(const AstP& a) {
    std::string n = a->name;
    if ((n == "count") && (a->a.empty() || a->a[0]->k == Ast::STAR)) return "count_star()";
    std::string arg = a->a.empty() ? "" : a->a[0]->text;
    return n + "(" + arg + ")";
  }

  // group key index of a column reference, -1 if none
  int group_index(int src, const Column* c) const {
    for (size_t i = 0; i < plan.group_keys.size(); ++i)
      if (plan.group_keys[i]->src == src && plan.group_keys[i]->col == c) return (int)i;
    return -1;
  }

  // ------------------------------------------------------------ statement
  void bind(const SelectStmt& st) {
    if (st.has_cte) fail(MTL_UNSUPPORTED, "CTEs are outside the offloaded subset");
    if (st.has_set_op) fail(MTL_UNSUPPORTED, "set operations are outside the offloaded subset");
    if (st.distinct) fail(MTL_UNSUPPORTED, "SELECT DISTINCT is outside the offloaded subset");
    if (st.has_having) fail(MTL_UNSUPPORTED, "HAVING is outside the offloaded subset");
    if (st.has_offset) fail(MTL_UNSUPPORTED, "OFFSET is outside the offloaded subset");
    plan.limit = st.limit;

    if (st.from.empty()) {
      bind_constant(st);
      return;
    }
    // sources and explicit joins
    std::vector<AstP> on_conds;
    for (size_t f = 0; f < st.from.size(); ++f) {
      add_source(st.from[f]);
      for (const JoinClause& j : st.joins[f]) {
        if (j.kind != "inner")
          fail(MTL_UNSUPPORTED, "outer and cross joins are outside the offloaded subset (" + j.kind + " join)");
        add_source(j.right);
        on_conds.push_back(j.on);
      }
    }
    if (plan.sources.size() > (size_t)kMaxSrc) fail(MTL_UNSUPPORTED, "too many tables in one query");
    for (auto& c : on_conds) conjunct(c);
    if (st.where) conjunct(st.where);

    // aggregate detection
    bool any_agg = false;
    for (auto& it : st.items)
      if (!it.star && contains_agg(it.expr)) any_agg = true;
    plan.is_agg = any_agg || !st.group_by.empty();

    if (plan.is_agg) {
      for (auto& g : st.group_by) {
        AstP ge = g;
        if (ge->k == Ast::INT) {
          long idx = strtol(ge->name.c_str(), nullptr, 10);
          if (idx < 1 || idx > (long)st.items.size()) fail(MTL_INVALID, "GROUP BY position out of range");
          ge = st.items[idx - 1].expr;
        } else if (ge->k == Ast::COL && ge->table.empty()) {
          // GROUP BY alias
          bool is_col = false;
          for (auto& s : plan.sources)
            if (s.table->find(ge->name)) is_col = true;
          if (!is_col)
            for (auto& it : st.items)
              if (!it.star && it.alias == ge->name) ge = it.expr;
        }
        if (ge->k != Ast::COL) fail(MTL_UNSUPPORTED, "GROUP BY on an expression is outside the offloaded subset");
        BExprP e = bind_expr(ge);
        if (group_index(e->src, e->col) < 0) plan.group_keys.push_back(e);
      }
      if (plan.group_keys.size() > (size_t)kMaxKeys) fail(MTL_UNSUPPORTED, "more than 4 GROUP BY keys");
      for (auto& it : st.items) {
        if (it.star) fail(MTL_INVALID, "SELECT * with GROUP BY");
        BOut o;
        if (it.expr->k == Ast::FUNC && is_agg_name(it.expr->name)) {
          o.agg_idx = bind_agg(it.expr);
          o.type = plan.aggs[o.agg_idx].result;
          o.name = it.alias.empty() ? agg_default_name(it.expr) : it.alias;
        } else if (it.expr->k == Ast::COL) {
          BExprP e = bind_expr(it.expr);
          int gi = group_index(e->src, e->col);
          if (gi < 0)
            fail(MTL_INVALID, "column \"" + it.expr->name +
                                  "\" must appear in the GROUP BY clause or be used in an aggregate function");
          o.group_idx = gi;
          o.type = e->type;
          o.name = it.alias.empty() ? it.expr->name : it.alias;
          if (e->col->type.t == MTL_T_VARCHAR) o.dict = &e->col->dict;
        } else {
          fail(MTL_UNSUPPORTED, "expressions over aggregates are outside the offloaded subset");
        }
        plan.outputs.push_back(o);
      }
    } else {
      for (auto& it : st.items) {
        if (it.star) {
          for (size_t s = 0; s < plan.sources.size(); ++s) {
            for (auto& c : plan.sources[s].table->cols) {
              BOut o;
              auto e = std::make_shared<BExpr>();
              e->k = BExpr::COL;
              e->src = (int)s;
              e->col = c.get();
              e->type = c->type;
              e->ptype = storage_ptype(c->type);
              o.expr = e;
              o.type = c->type;
              o.name = c->name;
              if (c->type.t == MTL_T_VARCHAR) o.dict = &c->dict;
              plan.outputs.push_back(o);
            }
          }
          continue;
        }
        BOut o;
        if (it.expr->k == Ast::STR) fail(MTL_UNSUPPORTED, "string literal outputs are outside the offloaded subset");
        o.expr = bind_expr(it.expr);
        o.type = o.expr->type;
        o.name = it.alias.empty() ? (it.expr->k == Ast::COL ? it.expr->name : it.expr->text) : it.alias;
        if (o.expr->k == BExpr::COL && o.expr->col->type.t == MTL_T_VARCHAR) o.dict = &o.expr->col->dict;
        else if (o.type.t == MTL_T_VARCHAR) fail(MTL_UNSUPPORTED, "VARCHAR expressions");
        plan.outputs.push_back(o);
      }
    }
    if (plan.outputs.size() > (size_t)kMaxProgs - 2) fail(MTL_UNSUPPORTED, "too many output columns");
    bind_order(st);
    plan.grouped_topk = plan.is_agg && !plan.group_keys.empty() && !plan.order.empty() && plan.limit >= 0;
  }

  void add_source(const TableRef& r) {
    std::lock_guard<std::recursive_mutex> g(ctx.mu);
    auto it = ctx.tables.find(r.name);
    if (it == ctx.tables.end())
      fail(MTL_UNSUPPORTED, "table \"" + r.name + "\" is not registered with gpu_register_table");
    Source s;
    s.name = r.name;
    s.alias = r.alias;
    s.table = it->second;
    plan.sources.push_back(s);
  }

  void bind_order(const SelectStmt& st) {
    for (const OrderItem& oi : st.order_by) {
      const AstP& a = oi.expr;
      int idx = -1;
      if (a->k == Ast::INT) {
        long k = strtol(a->name.c_str(), nullptr, 10);
        if (k < 1 || k > (long)plan.outputs.size()) fail(MTL_INVALID, "ORDER BY position out of range");
        idx = (int)k - 1;
      } else if (a->k == Ast::COL && a->table.empty()) {
        for (size_t i = 0; i < plan.outputs.size(); ++i)
          if (!plan.outputs[i].hidden && plan.outputs[i].name == a->name) {
            idx = (int)i;
            break;
          }
      }
      if (idx < 0 && a->k == Ast::COL) {
        auto [s, c] = resolve(*a);
        for (size_t i = 0; i < plan.outputs.size(); ++i) {
          const BOut& o = plan.outputs[i];
          if (plan.is_agg && o.group_idx >= 0 && plan.group_keys[o.group_idx]->src == s &&
              plan.group_keys[o.group_idx]->col == c) {
            idx = (int)i;
            break;
          }
          if (!plan.is_agg && o.expr && o.expr->k == BExpr::COL && o.expr->src == s && o.expr->col == c) {
            idx = (int)i;
            break;
          }
        }
        if (idx < 0) {
          BOut o;
          o.hidden = true;
          if (plan.is_agg) {
            int gi = group_index(s, c);
            if (gi < 0) fail(MTL_INVALID, "ORDER BY column must appear in the GROUP BY clause");
            o.group_idx = gi;
            o.type = c->type;
          } else {
            o.expr = bind_expr(a);
            o.type = o.expr->type;
          }
          o.name = a->name;
          if (c->type.t == MTL_T_VARCHAR) o.dict = &c->dict;
          plan.outputs.push_back(o);
          idx = (int)plan.outputs.size() - 1;
        }
      }
      if (idx < 0 && a->k == Ast::FUNC && is_agg_name(a->name) && plan.is_agg) {
        int ai = bind_agg(a);
        for (size_t i = 0; i < plan.outputs.size(); ++i)
          if (plan.outputs[i].agg_idx == ai) idx = (int)i;
        if (idx < 0) {
          BOut o;
          o.hidden = true;
          o.agg_idx = ai;
          o.type = plan.aggs[ai].result;
          o.name = a->text;
          plan.outputs.push_back(o);
          idx = (int)plan.outputs.size() - 1;
        }
      }
      if (idx < 0 && !plan.is_agg) {
        BOut o;
        o.hidden = true;
        o.expr = bind_expr(a);
        o.type = o.expr->type;
        o.name = a->text;
        plan.outputs.push_back(o);
        idx = (int)plan.outputs.size() - 1;
      }
      if (idx < 0) fail(MTL_UNSUPPORTED, "ORDER BY expression '" + a->text + "' is outside the offloaded subset");
      BOrder ob;
      ob.out = idx;
      ob.desc = oi.desc;
      plan.order.push_back(ob);
    }
    if (plan.order.size() > (size_t)kMaxOrder) fail(MTL_UNSUPPORTED, "too many ORDER BY keys");
  }

  // SELECT without FROM: constants only (evaluated on the host).
  void bind_constant(const SelectStmt& st) {
    plan.constant_only = true;
    for (auto& it : st.items) {
      if (it.star) fail(MTL_INVALID, "SELECT * with no tables specified is not valid");
      BOut o;
      if (it.expr->k == Ast::STR) {
        fail(MTL_UNSUPPORTED, "string constants are outside the offloaded subset");
      }
      o.expr = bind_expr(it.expr);
      if (o.expr->k != BExpr::CONST) fail(MTL_UNSUPPORTED, "non-constant expression without FROM");
      o.type = o.expr->type;
      o.name = it.alias.empty() ? it.expr->text : it.alias;
      plan.outputs.push_back(o);
    }
  }
};

}  // namespace

BoundPlan bind_select(Ctx& ctx, const SelectStmt& st) {
  BoundPlan plan;
  Binder b{ctx, plan};
  b.bind(st);
  return plan;
}

}  // namespace mtl
