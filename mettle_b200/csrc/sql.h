// sql.h — SQL front-end for the offloaded subset: tokens -> AST.
//
// Covers what the reference's sqlparser-based front-end accepts
// (src/plan/parser.rs:20-120): one SELECT with INNER / comma joins, an
// AND-only WHERE with comparisons and BETWEEN, DATE literals, + - *,
// SUM/COUNT/MIN/MAX/AVG, GROUP BY, ORDER BY and a numeric LIMIT; plus
// TIMESTAMP literals (which the reference cannot type) and the shapes it
// rejects (CTE, OR, outer joins, HAVING, DISTINCT, subqueries) parsed far
// enough to be reported as unsupported.
#pragma once
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace mtl {

struct SqlError : std::runtime_error {
  explicit SqlError(const std::string& m) : std::runtime_error(m) {}
};

struct Ast;
using AstP = std::shared_ptr<Ast>;

struct Ast {
  enum Kind { COL, INT, DEC, STR, DATE, TS, BIN, CMP, AND, OR, NOT, BETWEEN, FUNC, NEG, STAR, UNSUPPORTED };
  Kind k = COL;
  std::string table;  // COL: qualifier (lowercase) or ""
  std::string name;   // COL: column; FUNC: lowercase name; INT/DEC/STR/DATE/TS: literal text
  char op = 0;        // BIN: '+', '-', '*', '/'
  int cmp = 0;        // CMP: CmpOp
  bool distinct = false;
  bool negated = false;
  std::vector<AstP> a;
  std::string text;   // source text of the expression (result column naming)
};

struct SelectItem {
  AstP expr;
  std::string alias;
  bool star = false;
};

struct TableRef {
  std::string name;   // lowercase
  std::string alias;  // lowercase, "" when none
};

struct JoinClause {
  TableRef right;
  std::string kind;  // "inner", "left", "right", "full", "cross"
  AstP on;
};

struct OrderItem {
  AstP expr;
  bool desc = false;
};

struct SelectStmt {
  bool has_cte = false;
  bool distinct = false;
  bool has_having = false;
  bool has_offset = false;
  bool has_set_op = false;
  bool has_subquery = false;
  std::vector<SelectItem> items;
  std::vector<TableRef> from;                 // first table of each FROM item
  std::vector<std::vector<JoinClause>> joins; // joins chained onto each FROM item
  AstP where;
  std::vector<AstP> group_by;
  std::vector<OrderItem> order_by;
  int64_t limit = -1;
};

// Parses one statement; throws SqlError on malformed SQL.
SelectStmt parse_sql(const std::string& sql);

// Civil date <-> days since 1970-01-01 (the civil algorithm of
// src/plan/parser.rs:426-449).
int32_t days_from_civil(int32_t y, int32_t m, int32_t d);
void civil_from_days(int32_t z, int32_t* y, int32_t* m, int32_t* d);
// 'YYYY-MM-DD' -> days; false when malformed.
bool parse_date(const std::string& s, int32_t* days);
// 'YYYY-MM-DD[ HH:MM:SS[.ffffff]]' -> microseconds since epoch.
bool parse_timestamp(const std::string& s, int64_t* micros);

}  // namespace mtl
