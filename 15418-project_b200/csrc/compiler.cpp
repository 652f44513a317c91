// JSONPath -> byte IR compiler (host code).
//
// Same grammar, IR and error behaviour as the reference's QueryParser
// (src/gpjson/query/query_compiler.cpp:14-465): a recursive-descent parser
// over "$", ".name", "['name']", "[i]", "[i,j,...]", "[a:b]", "[:b]", "[-i]",
// "[-i:]" and "[?(@ == "x")]", emitting LEB128 operands
// (query_compiler.cpp:20-26) and counting result slots and levels the same
// way.  Queries in the reference's syntax compile to the reference's IR byte
// for byte.  Extensions (the reference rejects all of them):
//  * "[*]" with a wildcard limit K > 0: the open slice "[0:]" below (the
//    reference rejects "[*]", query_compiler.cpp:287-289);
//  * "..name" as the last step, with a wildcard limit K > 0: every member
//    named `name` inside the current value at any indexed level, in document
//    order, into K result slots (opcode 0x0B; query_compiler.cpp:202-204);
//  * numeric filters "[?(@<path> <op> <number>)]" with op one of == != < <=
//    > >= (opcode 0x0A: exact decimal comparison), and "!=" ... the filter
//    of the reference takes only == "string" (query_compiler.cpp:366-391);
//  * slices counted from the end: "[-a:-b]" (the reverse indexes a .. b+1,
//    reference IR only), and, with a wildcard limit K > 0, the open slices
//    "[a:]", "[a:-b]" and "[:-b]": an element-count check (opcode 0x0C,
//    raises the overflow status when the slice holds more than K elements)
//    and K forward branches as in "[a:a+K]", each checking that its element
//    exists and is followed by b more (opcode 0x0D; an empty array has no
//    element 0, where "[0]" of the reference stores the closing bracket).  The reference parses "[-a:" only
//    as "[-a:]" and rejects the others (query_compiler.cpp:256-286).
#include "compiler.hpp"

#include <algorithm>
#include <cctype>
#include <sstream>

namespace gpjb {
namespace {

enum Op : uint8_t {
  kEnd = 0,
  kStoreResult = 1,
  kMoveUp = 2,
  kMoveDown = 3,
  kMoveToKey = 4,
  kMoveToIndex = 5,
  kMoveToIndexReverse = 6,
  kMark = 7,
  kReset = 8,
  kStringEquals = 9,
  kNumberCompare = 10,  // extension: cmp byte, varint length, number text
  kDescendKey = 11,     // extension: varint length, key bytes
  kExpectAtMost = 12,   // extension: varint element limit
  kExpectFollowing = 13,  // extension: varint count of elements that must follow
};

// Comparators of kNumberCompare.
enum Cmp : uint8_t { kEq = 0, kNe = 1, kLt = 2, kLe = 3, kGt = 4, kGe = 5 };

// Levels a "..name" query asks the index for: every level the executor
// allows (max_depth < kMaxQueryLevels, query_executor_host.cu:129-131).
constexpr uint64_t kDescendLevels = 15;

class Emitter {
 public:
  void op(Op o) { bytes.push_back(uint8_t(o)); }
  void varint(uint64_t v) {
    while (v & ~uint64_t(0x7F)) {
      bytes.push_back(uint8_t((v & 0x7F) | 0x80));
      v >>= 7;
    }
    bytes.push_back(uint8_t(v & 0x7F));
  }
  void string(const std::string &s) {
    varint(s.size());
    bytes.insert(bytes.end(), s.begin(), s.end());
  }
  // IRBuilder bookkeeping (query_compiler.cpp:38-93)
  void property(const std::string &name) { op(kMoveToKey); string(name); }
  void index(uint64_t i) { op(kMoveToIndex); varint(i); }
  void reverse_index(uint64_t i) { op(kMoveToIndexReverse); varint(i); }
  void down() { op(kMoveDown); ++level; }
  void up() {
    op(kMoveUp);
    if (level > 0) --level;
  }
  void store() { op(kStoreResult); ++stores; }

  std::vector<uint8_t> bytes;
  uint64_t level = 0;
  uint64_t stores = 0;
};

// Cursor over the query text; `pos` is the index of the last consumed char
// (starts at -1), as in QueryScanner (query_compiler.cpp:95-171).
class Cursor {
 public:
  explicit Cursor(const std::string &t) : text(t) {}
  bool has_next() const { return pos + 1 < int64_t(text.size()); }
  char next() {
    if (!has_next()) throw fail(GPJ_ERR_MALFORMED_QUERY, "Expected character, got EOF");
    return text[size_t(++pos)];
  }
  char peek() const {
    if (!has_next()) throw fail(GPJ_ERR_MALFORMED_QUERY, "Expected character, got EOF");
    return text[size_t(pos + 1)];
  }
  void expect(char c) {
    const char a = next();
    if (a != c) {
      std::ostringstream m;
      m << "Expected character '" << c << "', got '" << a << "'";
      throw fail(GPJ_ERR_MALFORMED_QUERY, m.str());
    }
  }
  bool skip(char c) {
    if (!has_next() || peek() != c) return false;
    ++pos;
    return true;
  }
  std::string slice(int64_t start, int64_t end) const {
    if (end < start) return {};
    return text.substr(size_t(start + 1), size_t(end - start));
  }
  CompileError fail(int code, const std::string &msg) const {
    std::ostringstream m;
    m << msg << " at " << (pos + 1);
    if (pos + 1 < int64_t(text.size())) m << " ('" << text[size_t(pos + 1)] << "')";
    return CompileError{code, m.str()};
  }

  const std::string &text;
  int64_t pos = -1;
  std::vector<int64_t> marks;
};

class Parser {
 public:
  Parser(const std::string &q, uint64_t wildcard_limit)
      : cur(q), wildcard(wildcard_limit) {}

  CompiledIr run() {
    cur.expect('$');
    next_expression();
    if (!descended) ir.store();  // "..name" stores its own matches
    ir.op(kEnd);
    CompiledIr out;
    out.ir = std::move(ir.bytes);
    out.max_depth = max_level;
    out.num_result_slots = ir.stores;
    return out;
  }

 private:
  void next_expression() {
    if (!cur.has_next()) return;
    switch (cur.peek()) {
    case '.': dot(); break;
    case '[': bracket(); break;
    case ' ': return;
    case '=':
    case '!':
    case '<':
    case '>':
      if (in_filter > 0) return;  // the comparison of a filter follows its path
      [[fallthrough]];
    default: throw cur.fail(GPJ_ERR_UNSUPPORTED_QUERY, "Unsupported expression type");
    }
  }

  void dot() {
    cur.expect('.');
    if (cur.peek() == '.') {
      if (wildcard == 0 || in_filter > 0)
        throw cur.fail(GPJ_ERR_UNSUPPORTED_QUERY, "Unsupported recursive descent");
      descend();
      return;
    }
    const std::string name = read_property();
    if (name.empty()) throw cur.fail(GPJ_ERR_MALFORMED_QUERY, "Unexpected empty property");
    property(name);
    if (cur.has_next()) next_expression();
  }

  void bracket() {
    cur.expect('[');
    const char c = cur.peek();
    if (c == '\'' || c == '"') {
      const std::string name = read_quoted();
      if (name.empty()) throw cur.fail(GPJ_ERR_MALFORMED_QUERY, "Unexpected empty property");
      property(name);
    } else if (std::isdigit(static_cast<unsigned char>(c))) {
      const uint64_t i = read_integer([](char e) { return e == ']' || e == ':' || e == ','; });
      switch (cur.peek()) {
      case ':': {
        cur.expect(':');
        if (wildcard > 0 && (cur.peek() == ']' || cur.peek() == '-')) {
          open_slice(i);  // "[a:]", "[a:-b]"
          return;
        }
        const uint64_t end = read_integer([](char e) { return e == ']'; });
        cur.expect(']');
        range(i, end, false);
        return;
      }
      case ',': {
        std::vector<uint64_t> list{i};
        while (cur.peek() == ',') {
          cur.expect(',');
          if (!std::isdigit(static_cast<unsigned char>(cur.peek()))) {
            std::ostringstream m;
            m << "Expected digit, got '" << cur.peek() << "'";
            throw cur.fail(GPJ_ERR_MALFORMED_QUERY, m.str());
          }
          list.push_back(read_integer([](char e) { return e == ',' || e == ']'; }));
        }
        cur.expect(']');
        multiple(list);
        return;
      }
      case ']':
        ir.index(i);
        ir.down();
        ++max_level;
        break;
      default:
        throw cur.fail(GPJ_ERR_MALFORMED_QUERY, "Unexpected character in index expression");
      }
    } else if (c == ':') {
      cur.expect(':');
      if (wildcard > 0 && cur.peek() == '-') {
        open_slice(0);  // "[:-b]"
        return;
      }
      if (!std::isdigit(static_cast<unsigned char>(cur.peek())))
        throw cur.fail(GPJ_ERR_MALFORMED_QUERY, "Unexpected character in index, expected an integer");
      const uint64_t end = read_integer([](char e) { return e == ']'; });
      cur.expect(']');
      range(0, end, false);
      return;
    } else if (c == '-') {
      cur.expect('-');
      if (std::isdigit(static_cast<unsigned char>(cur.peek()))) {
        const uint64_t i = read_integer([](char e) { return e == ']' || e == ':'; });
        if (i == 0) throw cur.fail(GPJ_ERR_MALFORMED_QUERY, "Invalid reverse index 0");
        if (cur.peek() == ']') {
          ir.reverse_index(i);
          ir.down();
          ++max_level;
        } else {
          cur.expect(':');
          if (cur.peek() == '-') {
            // "[-a:-b]": the reverse indexes a .. b+1
            cur.expect('-');
            const uint64_t b = read_integer([](char e) { return e == ']'; });
            if (b == 0) throw cur.fail(GPJ_ERR_MALFORMED_QUERY, "Invalid reverse index 0");
            if (b >= i) throw cur.fail(GPJ_ERR_MALFORMED_QUERY, "Empty index range");
            cur.expect(']');
            range(b, i, true);
            return;
          }
          cur.expect(']');
          range(0, i, true);
          return;
        }
      } else if (cur.peek() == '-') {
        throw cur.fail(GPJ_ERR_UNSUPPORTED_QUERY, "Unsupported last n elements of the array query");
      } else {
        throw cur.fail(GPJ_ERR_MALFORMED_QUERY, "Unexpected character in index, expected an integer");
      }
    } else if (c == '*') {
      if (wildcard == 0) throw cur.fail(GPJ_ERR_UNSUPPORTED_QUERY, "Unsupported wildcard expression");
      cur.expect('*');
      open_slice(0, false);  // "[0:]": no silent truncation of longer arrays
      return;
    } else if (c == '?') {
      filter();
    } else {
      throw cur.fail(GPJ_ERR_MALFORMED_QUERY,
                     "Unexpected character in index, expected a quoted string or integer");
    }
    cur.expect(']');
    if (cur.has_next()) next_expression();
  }

  // "[a:]" and "[a:-b]" with the wildcard limit K: elements a .. a+K-1, each
  // checked to exist and, for "[a:-b]", to be followed by at least b
  // elements; an array with more than a+K+b elements raises the overflow
  // status.  The cursor is after ':' ("[*]": after '*').
  void open_slice(uint64_t start, bool from_end = true) {
    uint64_t tail = 0;
    if (from_end && cur.skip('-')) {
      tail = read_integer([](char e) { return e == ']'; });
      if (tail == 0) throw cur.fail(GPJ_ERR_MALFORMED_QUERY, "Invalid reverse index 0");
    }
    cur.expect(']');
    ir.op(kExpectAtMost);
    ir.varint(start + wildcard + tail);
    range(start, start + wildcard, false, int64_t(tail));
  }

  void multiple(const std::vector<uint64_t> &list) {
    uint64_t mm = max_level;
    for (size_t b = 0; b < list.size(); ++b) mm = branch(list[b], b + 1 == list.size(), mm, false);
    max_level = mm + 1;
  }

  void range(uint64_t start, uint64_t end, bool reverse, int64_t follow = -1) {
    uint64_t mm = max_level;
    if (reverse) {
      for (uint64_t i = end; i > start; --i) mm = branch(i, i == start + 1, mm, true);
    } else {
      for (uint64_t i = start; i < end; ++i) mm = branch(i, i + 1 == end, mm, false, follow);
    }
    max_level = mm + 1;
  }

  // query_compiler.cpp:335-364: one IR branch per index; every branch but the
  // last stores its result and climbs back to where it started.
  uint64_t branch(uint64_t index, bool last, uint64_t mm, bool reverse, int64_t follow = -1) {
    const uint64_t start_level = ir.level;
    if (reverse) ir.reverse_index(index);
    else ir.index(index);
    if (follow >= 0) {
      ir.op(kExpectFollowing);
      ir.varint(uint64_t(follow));
    }
    ir.down();
    cur.marks.push_back(cur.pos);
    const uint64_t saved = max_level;
    if (cur.has_next()) next_expression();
    mm = std::max(mm, max_level);
    max_level = saved;
    if (!last) {
      ir.store();
      cur.pos = cur.marks.back();
      cur.marks.pop_back();
      const uint64_t end_level = ir.level;
      for (uint64_t l = start_level; l < end_level; ++l) ir.up();
    }
    return mm;
  }

  void filter() {
    cur.expect('?');
    cur.expect('(');
    cur.expect('@');
    ir.op(kMark);
    ++in_filter;
    next_expression();
    --in_filter;
    while (cur.has_next() && cur.peek() == ' ') cur.skip(' ');
    Cmp cmp = kEq;
    switch (cur.peek()) {
    case '=':
      cur.expect('=');
      cur.expect('=');
      break;
    case '!':
      cur.expect('!');
      cur.expect('=');
      cmp = kNe;
      break;
    case '<':
    case '>': {
      const bool lt = cur.next() == '<';
      const bool eq = cur.skip('=');
      cmp = lt ? (eq ? kLe : kLt) : (eq ? kGe : kGt);
      break;
    }
    default:
      throw cur.fail(GPJ_ERR_UNSUPPORTED_QUERY, "Unsupported character for expression");
    }
    while (cur.has_next() && cur.peek() == ' ') cur.skip(' ');
    const char v = cur.peek();
    if (v == '-' || std::isdigit(static_cast<unsigned char>(v))) {
      const std::string number = read_number();
      ir.op(kNumberCompare);
      ir.bytes.push_back(uint8_t(cmp));
      ir.string(number);
    } else if (cmp == kEq) {
      // the reference's string filter (and its error for anything else)
      const std::string value = read_quoted();
      ir.op(kStringEquals);
      ir.string("\"" + value + "\"");
    } else if (v == '\'' || v == '"') {
      throw cur.fail(GPJ_ERR_UNSUPPORTED_QUERY, "Unsupported comparison of a string");
    } else {
      read_number();  // throws: not a number
    }
    ir.op(kReset);
    cur.expect(')');
  }

  // "..name" (an extension): every member named `name` inside the current
  // value, at any level the index holds, stored in document order into the
  // wildcard limit's K result slots.  It must be the last step.
  void descend() {
    cur.expect('.');
    const std::string name = read_property();
    if (name.empty()) throw cur.fail(GPJ_ERR_MALFORMED_QUERY, "Unexpected empty property");
    if (cur.has_next())
      throw cur.fail(GPJ_ERR_UNSUPPORTED_QUERY, "Unsupported expression after a recursive descent");
    ir.op(kDescendKey);
    ir.string(name);
    ir.stores += wildcard;
    descended = true;
    max_level = std::max<uint64_t>(max_level, kDescendLevels);
  }

  // A JSON number (RFC 8259: -?(0|[1-9][0-9]*)(.[0-9]+)?([eE][+-]?[0-9]+)?),
  // ending at ')' or ' '.
  std::string read_number() {
    const int64_t start = cur.pos;
    while (cur.has_next() && cur.peek() != ')' && cur.peek() != ' ') cur.next();
    const std::string t = cur.slice(start, cur.pos);
    size_t i = 0;
    auto digits = [&]() {
      const size_t b = i;
      while (i < t.size() && std::isdigit(static_cast<unsigned char>(t[i]))) ++i;
      return i - b;
    };
    bool ok = true;
    if (i < t.size() && t[i] == '-') ++i;
    if (i < t.size() && t[i] == '0') ++i;
    else ok = ok && i < t.size() && t[i] >= '1' && t[i] <= '9' && digits() > 0;
    if (ok && i < t.size() && t[i] == '.') {
      ++i;
      ok = digits() > 0;
    }
    if (ok && i < t.size() && (t[i] == 'e' || t[i] == 'E')) {
      ++i;
      if (i < t.size() && (t[i] == '+' || t[i] == '-')) ++i;
      ok = digits() > 0;
    }
    if (!ok || i != t.size()) throw cur.fail(GPJ_ERR_MALFORMED_QUERY, "Invalid number");
    while (cur.has_next() && cur.peek() == ' ') cur.skip(' ');
    return t;
  }

  void property(const std::string &name) {
    ir.property(name);
    ir.down();
    ++max_level;
  }

  std::string read_property() {
    const int64_t start = cur.pos;
    while (cur.has_next()) {
      const char c = cur.peek();
      if (c == '.' || c == '[' || c == ' ') break;
      cur.next();
    }
    return cur.slice(start, cur.pos);
  }

  std::string read_quoted() {
    const char q = cur.next();
    if (q != '\'' && q != '"') throw cur.fail(GPJ_ERR_MALFORMED_QUERY, "Invalid quoted string");
    const int64_t start = cur.pos;
    bool escaped = false;
    while (cur.has_next()) {
      const char c = cur.peek();
      if (escaped) escaped = false;
      else if (c == '\\') escaped = true;
      else if (c == q) break;
      cur.next();
    }
    const int64_t end = cur.pos;
    cur.expect(q);
    return cur.slice(start, end);
  }

  template <class IsEnd>
  uint64_t read_integer(IsEnd is_end) {
    const int64_t start = cur.pos;
    while (cur.has_next()) {
      const char c = cur.peek();
      if (std::isdigit(static_cast<unsigned char>(c))) {
        cur.next();
        continue;
      }
      if (is_end(c)) break;
      throw cur.fail(GPJ_ERR_MALFORMED_QUERY, "Invalid integer");
    }
    const std::string digits = cur.slice(start, cur.pos);
    // std::stoull in the reference: empty -> invalid_argument, too large ->
    // out_of_range (neither is a GpJSONError there).
    if (digits.empty()) throw CompileError{GPJ_ERR_INVALID_ARGUMENT, "stoull"};
    uint64_t v = 0;
    for (char d : digits) {
      const uint64_t nv = v * 10u + uint64_t(d - '0');
      if (v > (~uint64_t(0) - uint64_t(d - '0')) / 10u) throw CompileError{GPJ_ERR_OUT_OF_RANGE, "stoull"};
      v = nv;
    }
    return v;
  }

  Cursor cur;
  Emitter ir;
  uint64_t max_level = 0;
  uint64_t wildcard;
  int in_filter = 0;
  bool descended = false;
};

}  // namespace

CompiledIr compile_query(const std::string &text, uint64_t wildcard_limit) {
  Parser p(text, wildcard_limit);
  return p.run();
}

}  // namespace gpjb
