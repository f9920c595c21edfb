// sql.cpp — tokenizer and recursive-descent parser for the offloaded SQL
// subset (see sql.h). Identifiers fold to lower case unless double quoted,
// as in DuckDB.
#include "sql.h"

#include <cctype>
#include <cstdlib>
#include <cstring>

#include "dev_types.h"

namespace mtl {

// ------------------------------------------------------------ dates
int32_t days_from_civil(int32_t y, int32_t m, int32_t d) {
  int32_t ay = y - (m <= 2);
  int32_t era = (ay >= 0 ? ay : ay - 399) / 400;
  int32_t yoe = ay - era * 400;
  int32_t mo = m + (m > 2 ? -3 : 9);
  int32_t doy = (153 * mo + 2) / 5 + d - 1;
  int32_t doe = yoe * 365 + yoe / 4 - yoe / 100 + doy;
  return era * 146097 + doe - 719468;
}

void civil_from_days(int32_t z, int32_t* y, int32_t* m, int32_t* d) {
  z += 719468;
  int32_t era = (z >= 0 ? z : z - 146096) / 146097;
  int32_t doe = z - era * 146097;
  int32_t yoe = (doe - doe / 1460 + doe / 36524 - doe / 146096) / 365;
  int32_t yy = yoe + era * 400;
  int32_t doy = doe - (365 * yoe + yoe / 4 - yoe / 100);
  int32_t mp = (5 * doy + 2) / 153;
  int32_t dd = doy - (153 * mp + 2) / 5 + 1;
  int32_t mm = mp + (mp < 10 ? 3 : -9);
  *y = yy + (mm <= 2);
  *m = mm;
  *d = dd;
}

static bool parse_int_field(const char*& p, int digits_min, int digits_max, int* out) {
  int v = 0, n = 0;
  while (isdigit((unsigned char)*p) && n < digits_max) {
    v = v * 10 + (*p - '0');
    ++p;
    ++n;
  }
  if (n < digits_min) return false;
  *out = v;
  return true;
}

static int days_in_month(int y, int m) {
  static const int dm[] = {31, 28, 31, 30, 31, 30, 31, 31, 30, 31, 30, 31};
  bool leap = (y % 4 == 0 && y % 100 != 0) || y % 400 == 0;
  return m == 2 && leap ? 29 : dm[m - 1];
}

bool parse_date(const std::string& s, int32_t* days) {
  const char* p = s.c_str();
  while (*p == ' ') ++p;
  bool neg = false;
  if (*p == '-') {
    neg = true;
    ++p;
  }
  int y, m, d;
  if (!parse_int_field(p, 1, 6, &y) || *p++ != '-') return false;
  if (!parse_int_field(p, 1, 2, &m) || *p++ != '-') return false;
  if (!parse_int_field(p, 1, 2, &d)) return false;
  while (*p == ' ') ++p;
  if (*p) return false;
  if (neg) y = -y;
  if (m < 1 || m > 12 || d < 1 || d > days_in_month(y, m)) return false;
  *days = days_from_civil(y, m, d);
  return true;
}

bool parse_timestamp(const std::string& s, int64_t* micros) {
  const char* p = s.c_str();
  while (*p == ' ') ++p;
  int y, m, d, hh = 0, mi = 0, ss = 0;
  int64_t frac = 0;
  if (!parse_int_field(p, 1, 6, &y) || *p++ != '-') return false;
  if (!parse_int_field(p, 1, 2, &m) || *p++ != '-') return false;
  if (!parse_int_field(p, 1, 2, &d)) return false;
  if (*p == ' ' || *p == 'T') {
    ++p;
    if (!parse_int_field(p, 1, 2, &hh) || *p++ != ':') return false;
    if (!parse_int_field(p, 1, 2, &mi) || *p++ != ':') return false;
    if (!parse_int_field(p, 1, 2, &ss)) return false;
    if (*p == '.') {
      ++p;
      int n = 0;
      while (isdigit((unsigned char)*p)) {
        if (n < 6) {
          frac = frac * 10 + (*p - '0');
          ++n;
        }
        ++p;
      }
      while (n < 6) {
        frac *= 10;
        ++n;
      }
    }
  }
  while (*p == ' ') ++p;
  if (*p) return false;
  if (m < 1 || m > 12 || d < 1 || d > days_in_month(y, m) || hh > 23 || mi > 59 || ss > 59) return false;
  int64_t days = days_from_civil(y, m, d);
  *micros = ((days * 24 + hh) * 60 + mi) * 60 * 1000000LL + ss * 1000000LL + frac;
  return true;
}

// ------------------------------------------------------------ tokenizer
namespace {

enum TokKind { T_END, T_IDENT, T_QIDENT, T_NUM, T_STR, T_SYM };

struct Tok {
  TokKind k;
  std::string v;  // identifiers lower-cased; symbols as text
  size_t pos;
};

std::vector<Tok> tokenize(const std::string& s) {
  std::vector<Tok> out;
  size_t i = 0, n = s.size();
  while (i < n) {
    char c = s[i];
    if (isspace((unsigned char)c)) {
      ++i;
      continue;
    }
    if (c == '-' && i + 1 < n && s[i + 1] == '-') {  // line comment
      while (i < n && s[i] != '\n') ++i;
      continue;
    }
    if (c == '/' && i + 1 < n && s[i + 1] == '*') {
      i += 2;
      while (i + 1 < n && !(s[i] == '*' && s[i + 1] == '/')) ++i;
      i += 2;
      continue;
    }
    size_t st = i;
    if (isalpha((unsigned char)c) || c == '_') {
      while (i < n && (isalnum((unsigned char)s[i]) || s[i] == '_')) ++i;
      std::string v = s.substr(st, i - st);
      for (auto& ch : v) ch = (char)tolower((unsigned char)ch);
      out.push_back({T_IDENT, v, st});
      continue;
    }
    if (c == '"') {
      std::string v;
      ++i;
      while (i < n) {
        if (s[i] == '"') {
          if (i + 1 < n && s[i + 1] == '"') {
            v += '"';
            i += 2;
            continue;
          }
          break;
        }
        v += s[i++];
      }
      if (i >= n) throw SqlError("unterminated quoted identifier");
      ++i;
      out.push_back({T_QIDENT, v, st});
      continue;
    }
    if (c == '\'') {
      std::string v;
      ++i;
      while (i < n) {
        if (s[i] == '\'') {
          if (i + 1 < n && s[i + 1] == '\'') {
            v += '\'';
            i += 2;
            continue;
          }
          break;
        }
        v += s[i++];
      }
      if (i >= n) throw SqlError("unterminated string literal");
      ++i;
      out.push_back({T_STR, v, st});
      continue;
    }
    if (isdigit((unsigned char)c) || (c == '.' && i + 1 < n && isdigit((unsigned char)s[i + 1]))) {
      while (i < n && (isdigit((unsigned char)s[i]) || s[i] == '.')) ++i;
      if (i < n && (s[i] == 'e' || s[i] == 'E')) {
        size_t j = i + 1;
        if (j < n && (s[j] == '+' || s[j] == '-')) ++j;
        if (j < n && isdigit((unsigned char)s[j])) {
          i = j;
          while (i < n && isdigit((unsigned char)s[i])) ++i;
        }
      }
      out.push_back({T_NUM, s.substr(st, i - st), st});
      continue;
    }
    static const char* two[] = {"<=", ">=", "<>", "!=", "==", "::", "||"};
    bool matched = false;
    for (const char* t : two) {
      if (i + 1 < n && s[i] == t[0] && s[i + 1] == t[1]) {
        out.push_back({T_SYM, std::string(t), st});
        i += 2;
        matched = true;
        break;
      }
    }
    if (matched) continue;
    if (strchr("(),.;*+-/%<>=", c)) {
      out.push_back({T_SYM, std::string(1, c), st});
      ++i;
      continue;
    }
    throw SqlError(std::string("unexpected character '") + c + "'");
  }
  out.push_back({T_END, "", n});
  return out;
}

const char* kReserved[] = {"select", "from",  "where", "group",  "by",      "order", "limit", "as",
                           "and",    "or",    "not",   "between", "join",   "inner", "left",  "right",
                           "full",   "outer", "cross", "on",      "asc",    "desc",  "distinct",
                           "having", "with",  "union", "except",  "intersect", "offset", "nulls",
                           "in",     "is",    "null",  "case",    "when",   "then",  "else", "end",
                           "like",   "exists", "qualify", "window", "using", "natural", "all"};

bool reserved(const std::string& v) {
  for (const char* r : kReserved)
    if (v == r) return true;
  return false;
}

class Parser {
 public:
  Parser(const std::string& sql) : src_(sql), t_(tokenize(sql)) {}

  SelectStmt statement() {
    SelectStmt st;
    if (is_kw("with")) {
      st.has_cte = true;
      // Skip the CTE list; the main SELECT is still parsed for diagnostics.
      next();
      int depth = 0;
      while (!at_end()) {
        if (is_sym("(")) ++depth;
        if (is_sym(")")) --depth;
        if (depth == 0 && is_kw("select")) break;
        next();
      }
    }
    select(st);
    while (is_sym(";")) next();
    if (!at_end()) {
      if (is_kw("union") || is_kw("except") || is_kw("intersect")) {
        st.has_set_op = true;
        return st;
      }
      throw SqlError("unexpected token '" + cur().v + "' after statement");
    }
    return st;
  }

 private:
  const std::string& src_;
  std::vector<Tok> t_;
  size_t p_ = 0;
  bool subquery_ = false;

  const Tok& cur() const { return t_[p_]; }
  bool at_end() const { return t_[p_].k == T_END; }
  void next() {
    if (!at_end()) ++p_;
  }
  bool is_kw(const char* k) const { return cur().k == T_IDENT && cur().v == k; }
  bool is_kw_at(size_t off, const char* k) const {
    return p_ + off < t_.size() && t_[p_ + off].k == T_IDENT && t_[p_ + off].v == k;
  }
  bool is_sym(const char* s) const { return cur().k == T_SYM && cur().v == s; }
  void expect_kw(const char* k) {
    if (!is_kw(k)) throw SqlError(std::string("expected ") + k + " near '" + cur().v + "'");
    next();
  }
  void expect_sym(const char* s) {
    if (!is_sym(s)) throw SqlError(std::string("expected '") + s + "' near '" + cur().v + "'");
    next();
  }
  bool accept_kw(const char* k) {
    if (is_kw(k)) {
      next();
      return true;
    }
    return false;
  }
  bool accept_sym(const char* s) {
    if (is_sym(s)) {
      next();
      return true;
    }
    return false;
  }
  std::string ident() {
    if (cur().k == T_QIDENT) {
      std::string v = cur().v;
      next();
      return v;
    }
    if (cur().k == T_IDENT && !reserved(cur().v)) {
      std::string v = cur().v;
      next();
      return v;
    }
    throw SqlError("expected identifier near '" + cur().v + "'");
  }
  bool at_ident() const { return cur().k == T_QIDENT || (cur().k == T_IDENT && !reserved(cur().v)); }

  void select(SelectStmt& st) {
    expect_kw("select");
    if (accept_kw("distinct")) st.distinct = true;
    accept_kw("all");
    // items
    for (;;) {
      SelectItem it;
      if (is_sym("*")) {
        next();
        it.star = true;
      } else {
        it.expr = expr();
        if (accept_kw("as")) {
          it.alias = ident();
        } else if (at_ident()) {
          it.alias = ident();
        } else if (cur().k == T_STR) {
          it.alias = cur().v;
          next();
        }
      }
      st.items.push_back(it);
      if (!accept_sym(",")) break;
    }
    if (accept_kw("from")) {
      for (;;) {
        st.from.push_back(table_ref());
        std::vector<JoinClause> joins;
        for (;;) {
          JoinClause jc;
          if (accept_kw("join")) {
            jc.kind = "inner";
          } else if (is_kw("inner") && is_kw_at(1, "join")) {
            next();
            next();
            jc.kind = "inner";
          } else if (is_kw("left") || is_kw("right") || is_kw("full")) {
            jc.kind = cur().v;
            next();
            accept_kw("outer");
            expect_kw("join");
          } else if (is_kw("cross") && is_kw_at(1, "join")) {
            next();
            next();
            jc.kind = "cross";
          } else if (is_kw("natural")) {
            throw SqlError("NATURAL JOIN is not supported");
          } else {
            break;
          }
          jc.right = table_ref();
          if (jc.kind != "cross") {
            if (accept_kw("using")) throw SqlError("JOIN ... USING is not supported");
            expect_kw("on");
            jc.on = expr();
          }
          joins.push_back(jc);
        }
        st.joins.push_back(joins);
        if (!accept_sym(",")) break;
      }
    }
    if (accept_kw("where")) st.where = expr();
    if (is_kw("group")) {
      next();
      expect_kw("by");
      for (;;) {
        st.group_by.push_back(expr());
        if (!accept_sym(",")) break;
      }
    }
    if (accept_kw("having")) {
      st.has_having = true;
      expr();
    }
    if (is_kw("qualify") || is_kw("window")) throw SqlError("QUALIFY/WINDOW are not supported");
    if (is_kw("order")) {
      next();
      expect_kw("by");
      for (;;) {
        OrderItem oi;
        oi.expr = expr();
        if (accept_kw("desc")) oi.desc = true;
        else accept_kw("asc");
        if (accept_kw("nulls")) {
          if (!accept_kw("first") && !accept_kw("last")) throw SqlError("expected FIRST or LAST");
        }
        st.order_by.push_back(oi);
        if (!accept_sym(",")) break;
      }
    }
    if (accept_kw("limit")) {
      if (cur().k != T_NUM) throw SqlError("LIMIT expects a number");
      char* end = nullptr;
      long long v = strtoll(cur().v.c_str(), &end, 10);
      if (*end || v < 0) throw SqlError("LIMIT expects a non-negative integer");
      st.limit = v;
      next();
    }
    if (accept_kw("offset")) {
      st.has_offset = true;
      next();
    }
    if (subquery_) st.has_subquery = true;
  }

  TableRef table_ref() {
    if (is_sym("(")) {
      subquery_ = true;
      throw SqlError("subqueries in FROM are not supported");
    }
    TableRef r;
    r.name = ident();
    while (accept_sym(".")) r.name = ident();  // schema.table -> table
    if (accept_kw("as")) r.alias = ident();
    else if (at_ident()) r.alias = ident();
    return r;
  }

  AstP mk(Ast::Kind k, size_t start) {
    auto a = std::make_shared<Ast>();
    a->k = k;
    (void)start;
    return a;
  }
  void set_text(AstP& a, size_t start_tok) {
    size_t b = t_[start_tok].pos;
    size_t e = p_ > 0 ? t_[p_ - 1].pos + token_len(t_[p_ - 1]) : b;
    if (e > src_.size()) e = src_.size();
    a->text = src_.substr(b, e > b ? e - b : 0);
  }
  size_t token_len(const Tok& t) const {
    if (t.k == T_STR) {
      // find the closing quote from the token start
      size_t i = t.pos + 1;
      while (i < src_.size()) {
        if (src_[i] == '\'') {
          if (i + 1 < src_.size() && src_[i + 1] == '\'') {
            i += 2;
            continue;
          }
          return i + 1 - t.pos;
        }
        ++i;
      }
      return src_.size() - t.pos;
    }
    if (t.k == T_QIDENT) {
      size_t i = t.pos + 1;
      while (i < src_.size() && src_[i] != '"') ++i;
      return i + 1 - t.pos;
    }
    return t.v.size();
  }

  AstP expr() { return or_expr(); }

  AstP or_expr() {
    size_t s0 = p_;
    AstP l = and_expr();
    while (accept_kw("or")) {
      AstP n = mk(Ast::OR, s0);
      n->a = {l, and_expr()};
      set_text(n, s0);
      l = n;
    }
    return l;
  }
  AstP and_expr() {
    size_t s0 = p_;
    AstP l = not_expr();
    while (accept_kw("and")) {
      AstP n = mk(Ast::AND, s0);
      n->a = {l, not_expr()};
      set_text(n, s0);
      l = n;
    }
    return l;
  }
  AstP not_expr() {
    size_t s0 = p_;
    if (accept_kw("not")) {
      AstP n = mk(Ast::NOT, s0);
      n->a = {not_expr()};
      set_text(n, s0);
      return n;
    }
    return cmp_expr();
  }
  AstP cmp_expr() {
    size_t s0 = p_;
    AstP l = add_expr();
    static const struct {
      const char* s;
      int op;
    } ops[] = {{"=", C_EQ}, {"==", C_EQ}, {"<", C_LT}, {"<=", C_LE}, {">", C_GT}, {">=", C_GE}, {"<>", C_NE}, {"!=", C_NE}};
    for (auto& o : ops) {
      if (is_sym(o.s)) {
        next();
        AstP n = mk(Ast::CMP, s0);
        n->cmp = o.op;
        n->a = {l, add_expr()};
        set_text(n, s0);
        return n;
      }
    }
    bool neg = false;
    if (is_kw("not") && is_kw_at(1, "between")) {
      next();
      neg = true;
    }
    if (accept_kw("between")) {
      AstP n = mk(Ast::BETWEEN, s0);
      n->negated = neg;
      AstP lo = add_expr();
      expect_kw("and");
      AstP hi = add_expr();
      n->a = {l, lo, hi};
      set_text(n, s0);
      return n;
    }
    if (is_kw("in") || is_kw("is") || is_kw("like") || (is_kw("not") && (is_kw_at(1, "in") || is_kw_at(1, "like")))) {
      // Parsed only to report the shape as unsupported.
      AstP n = mk(Ast::UNSUPPORTED, s0);
      n->name = cur().v;
      while (!at_end() && !is_kw("and") && !is_kw("or") && !is_sym(")") && !is_kw("group") && !is_kw("order") &&
             !is_kw("limit")) {
        if (is_sym("(")) {
          int depth = 0;
          do {
            if (is_sym("(")) ++depth;
            if (is_sym(")")) --depth;
            next();
          } while (!at_end() && depth > 0);
          continue;
        }
        next();
      }
      return n;
    }
    return l;
  }
  AstP add_expr() {
    size_t s0 = p_;
    AstP l = mul_expr();
    while (is_sym("+") || is_sym("-") || is_sym("||")) {
      char op = cur().v == "||" ? '|' : cur().v[0];
      next();
      AstP n = mk(Ast::BIN, s0);
      n->op = op;
      n->a = {l, mul_expr()};
      set_text(n, s0);
      l = n;
    }
    return l;
  }
  AstP mul_expr() {
    size_t s0 = p_;
    AstP l = unary();
    while (is_sym("*") || is_sym("/") || is_sym("%")) {
      char op = cur().v[0];
      next();
      AstP n = mk(Ast::BIN, s0);
      n->op = op;
      n->a = {l, unary()};
      set_text(n, s0);
      l = n;
    }
    return l;
  }
  AstP unary() {
    size_t s0 = p_;
    if (accept_sym("-")) {
      AstP n = mk(Ast::NEG, s0);
      n->a = {unary()};
      set_text(n, s0);
      return n;
    }
    if (accept_sym("+")) return unary();
    AstP e = primary();
    if (accept_sym("::")) {
      AstP n = mk(Ast::UNSUPPORTED, s0);
      n->name = "cast";
      ident();
      if (accept_sym("(")) {
        while (!at_end() && !is_sym(")")) next();
        expect_sym(")");
      }
      set_text(n, s0);
      return n;
    }
    return e;
  }
  AstP primary() {
    size_t s0 = p_;
    const Tok t = cur();
    if (t.k == T_NUM) {
      next();
      bool is_dec = t.v.find_first_of(".eE") != std::string::npos;
      AstP n = mk(is_dec ? Ast::DEC : Ast::INT, s0);
      n->name = t.v;
      set_text(n, s0);
      return n;
    }
    if (t.k == T_STR) {
      next();
      AstP n = mk(Ast::STR, s0);
      n->name = t.v;
      set_text(n, s0);
      return n;
    }
    if (t.k == T_SYM && t.v == "(") {
      next();
      if (is_kw("select")) {
        subquery_ = true;
        throw SqlError("subqueries are not supported");
      }
      AstP e = expr();
      expect_sym(")");
      set_text(e, s0);
      return e;
    }
    if (t.k == T_SYM && t.v == "*") {
      next();
      AstP n = mk(Ast::STAR, s0);
      set_text(n, s0);
      return n;
    }
    if (t.k == T_IDENT && (t.v == "date" || t.v == "timestamp") && t_[p_ + 1].k == T_STR) {
      next();
      AstP n = mk(t.v == "date" ? Ast::DATE : Ast::TS, s0);
      n->name = cur().v;
      next();
      set_text(n, s0);
      return n;
    }
    if (t.k == T_IDENT && (t.v == "case" || t.v == "exists" || t.v == "cast" || t.v == "null")) {
      AstP n = mk(Ast::UNSUPPORTED, s0);
      n->name = t.v;
      next();
      if (t.v == "case") {
        int depth = 1;
        while (!at_end() && depth > 0) {
          if (is_kw("case")) ++depth;
          if (is_kw("end")) --depth;
          next();
        }
      } else if (is_sym("(")) {
        int depth = 0;
        do {
          if (is_sym("(")) ++depth;
          if (is_sym(")")) --depth;
          next();
        } while (!at_end() && depth > 0);
      }
      set_text(n, s0);
      return n;
    }
    if (t.k == T_IDENT || t.k == T_QIDENT) {
      if (t.k == T_IDENT && reserved(t.v)) throw SqlError("unexpected keyword '" + t.v + "'");
      std::string first = t.v;
      next();
      if (t.k == T_IDENT && is_sym("(")) {
        next();
        AstP n = mk(Ast::FUNC, s0);
        n->name = first;
        if (accept_kw("distinct")) n->distinct = true;
        if (!is_sym(")")) {
          for (;;) {
            if (is_sym("*")) {
              size_t s1 = p_;
              next();
              AstP st = mk(Ast::STAR, s1);
              set_text(st, s1);
              n->a.push_back(st);
            } else {
              n->a.push_back(expr());
            }
            if (!accept_sym(",")) break;
          }
        }
        expect_sym(")");
        if (is_kw("over") || is_kw("filter")) throw SqlError("window and FILTER aggregates are not supported");
        set_text(n, s0);
        return n;
      }
      AstP n = mk(Ast::COL, s0);
      if (accept_sym(".")) {
        if (is_sym("*")) throw SqlError("qualified * is not supported");
        n->table = first;
        n->name = ident();
        while (accept_sym(".")) {  // schema.table.column
          n->table = n->name;
          n->name = ident();
        }
      } else {
        n->name = first;
      }
      set_text(n, s0);
      return n;
    }
    throw SqlError("unexpected token '" + t.v + "'");
  }
};

}  // namespace

SelectStmt parse_sql(const std::string& sql) {
  Parser p(sql);
  return p.statement();
}

}  // namespace mtl
