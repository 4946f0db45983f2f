// The reference's YAML input deck read inside the library (host code only):
// InputSettings::from_yaml_str (settings.rs:27-511) on a small YAML reader of
// the block and flow forms decks use, with plain scalars typed by the YAML 1.2
// core rules of the reference's reader (serde_yaml_ng 0.10). The schema
// checks, defaults and error kinds are those of the Python front door
// (pwgpu/deck.py), which the tests hold this reader to.
#include <cctype>
#include <charconv>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <utility>
#include <vector>

#include "handle.hpp"
#include "../../include/pwgpu_deck.h"

namespace {

using pwgpu::fail;

struct ParseError {
  std::string msg;
};
struct InvalidParam {
  std::string msg;
};

[[noreturn]] void perr(const std::string& m) { throw ParseError{m}; }

// ---------------------------------------------------------------------------
// YAML subset: nodes
// ---------------------------------------------------------------------------

struct Node {
  enum Kind { kNull, kScalar, kSeq, kMap } kind = kNull;
  std::string text;  // scalar text
  bool plain = true;
  std::vector<Node> items;
  std::vector<std::pair<std::string, Node>> entries;

  const Node* get(const std::string& k) const {
    for (auto& e : entries)
      if (e.first == k) return &e.second;
    return nullptr;
  }
};

// typed value of a scalar node
struct Value {
  enum Type { kNone, kBool, kInt, kFloat, kStr } type = kNone;
  bool b = false;
  long long i = 0;
  double f = 0.0;
  std::string s;
};

bool all_digits(const std::string& s, int base) {
  if (s.empty()) return false;
  for (char c : s) {
    int d = std::isdigit((unsigned char)c) ? c - '0'
            : (c >= 'a' && c <= 'f')       ? c - 'a' + 10
            : (c >= 'A' && c <= 'F')       ? c - 'A' + 10
                                           : 99;
    if (d >= base) return false;
  }
  return true;
}

bool is_decimal_float(const std::string& v) {
  // [-+]?([0-9]+\.?[0-9]*|\.[0-9]+)([eE][-+]?[0-9]+)?
  size_t i = 0, n = v.size();
  if (i < n && (v[i] == '+' || v[i] == '-')) ++i;
  size_t d0 = i;
  while (i < n && std::isdigit((unsigned char)v[i])) ++i;
  bool int_digits = i > d0;
  bool frac_digits = false;
  if (i < n && v[i] == '.') {
    ++i;
    size_t f0 = i;
    while (i < n && std::isdigit((unsigned char)v[i])) ++i;
    frac_digits = i > f0;
  }
  if (!int_digits && !frac_digits) return false;
  if (i < n && (v[i] == 'e' || v[i] == 'E')) {
    ++i;
    if (i < n && (v[i] == '+' || v[i] == '-')) ++i;
    size_t e0 = i;
    while (i < n && std::isdigit((unsigned char)v[i])) ++i;
    if (i == e0) return false;
  }
  return i == n;
}

Value core_scalar(const std::string& v) {
  Value r;
  if (v.empty() || v == "~" || v == "null" || v == "Null" || v == "NULL") return r;
  if (v == "true" || v == "True" || v == "TRUE") { r.type = Value::kBool; r.b = true; return r; }
  if (v == "false" || v == "False" || v == "FALSE") { r.type = Value::kBool; r.b = false; return r; }
  r.type = Value::kStr;
  r.s = v;
  std::string unsig = (!v.empty() && v[0] == '+') ? v.substr(1) : v;
  if (v[0] == '+' && !unsig.empty() && (unsig[0] == '+' || unsig[0] == '-')) return r;
  static const std::pair<const char*, int> radix[] = {{"0x", 16}, {"0o", 8}, {"0b", 2}};
  for (auto& p : radix) {
    if (unsig.rfind(p.first, 0) == 0) {
      const std::string digits = unsig.substr(2);
      if (!all_digits(digits, p.second) || digits.size() > 15) return r;
      r.type = Value::kInt;
      r.i = std::stoll(digits, nullptr, p.second);
      return r;
    }
  }
  std::string mag = unsig;
  while (!mag.empty() && mag[0] == '-') mag = mag.substr(1);
  if (mag.size() > 1 && mag[0] == '0' && all_digits(mag, 10)) return r;
  {
    size_t k = (v[0] == '+' || v[0] == '-') ? 1 : 0;
    if (k < v.size() && all_digits(v.substr(k), 10)) {
      if (v.size() - k > 18) return r;  // beyond int64: the schema's integers never reach this
      r.type = Value::kInt;
      r.i = std::stoll(v);
      return r;
    }
  }
  if (unsig == ".inf" || unsig == ".Inf" || unsig == ".INF") { r.type = Value::kFloat; r.f = INFINITY; return r; }
  if (v == "-.inf" || v == "-.Inf" || v == "-.INF") { r.type = Value::kFloat; r.f = -INFINITY; return r; }
  if (v == ".nan" || v == ".NaN" || v == ".NAN") { r.type = Value::kFloat; r.f = NAN; return r; }
  if (is_decimal_float(v)) {
    const double x = std::strtod(v.c_str(), nullptr);
    if (std::isfinite(x)) { r.type = Value::kFloat; r.f = x; }
  }
  return r;
}

Value typed(const Node* n) {
  Value r;
  if (!n || n->kind == Node::kNull) return r;
  if (n->kind != Node::kScalar) { r.type = Value::kStr; r.s = "<collection>"; return r; }
  if (!n->plain) { r.type = Value::kStr; r.s = n->text; return r; }
  return core_scalar(n->text);
}

// ---------------------------------------------------------------------------
// YAML subset: reader
// ---------------------------------------------------------------------------

struct Line {
  int indent;
  std::string text;
  int no;
};

std::string rtrim(std::string s) {
  while (!s.empty() && (s.back() == ' ' || s.back() == '\t' || s.back() == '\r' || s.back() == '\n')) s.pop_back();
  return s;
}
std::string trim(const std::string& s) {
  size_t a = 0;
  while (a < s.size() && (s[a] == ' ' || s[a] == '\t' || s[a] == '\n')) ++a;
  return rtrim(s.substr(a));
}

// Scan of one line's text outside quoted scalars: a quote or a `[` / `{`
// opens only where a scalar or collection can start (at the start, or after
// one of `[ { , : - ?` and blanks); a `#` starts a comment after a blank or
// right after a closed quote, bracket or comma. Returns the text before the
// comment; *depth receives the open-bracket count at the end.
std::string scan_line(const std::string& s, int* depth) {
  bool sq = false, dq = false;
  char last = '\0';  // last non-blank character outside quotes
  bool closed = false;  // the previous character closed a quote, a bracket or was a comma
  int d = 0;
  for (size_t i = 0; i < s.size(); ++i) {
    const char c = s[i];
    if (dq) {
      if (c == '\\') ++i;
      else if (c == '"') { dq = false; last = c; closed = true; }
      continue;
    }
    if (sq) {
      if (c == '\'') {
        if (i + 1 < s.size() && s[i + 1] == '\'') { ++i; continue; }
        sq = false; last = c; closed = true;
      }
      continue;
    }
    const bool can_open = last == '\0' || std::strchr("[{,:-?", last) != nullptr;
    if (c == '#' && (i == 0 || s[i - 1] == ' ' || s[i - 1] == '\t' || s[i - 1] == '\n' || closed)) {
      if (depth) *depth = d;
      return s.substr(0, i);
    }
    closed = false;
    if (c == ' ' || c == '\t' || c == '\n') continue;
    if ((c == '"' || c == '\'') && can_open) {
      (c == '"' ? dq : sq) = true;
    } else if ((c == '[' || c == '{') && can_open) {
      ++d;
    } else if ((c == ']' || c == '}') && d > 0) {
      --d;
      closed = true;
    } else if (c == ',' && d > 0) {
      closed = true;
    }
    last = c;
  }
  if (depth) *depth = d;
  return s;
}

std::string strip_comment(const std::string& s) { return scan_line(s, nullptr); }

int bracket_depth(const std::string& s) {
  int d = 0;
  scan_line(s, &d);
  return d;
}

std::vector<Line> split_lines(const std::string& text) {
  std::vector<Line> out;
  size_t p = 0;
  int no = 0;
  bool started = false;
  while (p <= text.size()) {
    size_t e = text.find('\n', p);
    if (e == std::string::npos) e = text.size();
    std::string raw = text.substr(p, e - p);
    p = e + 1;
    ++no;
    std::string s = rtrim(strip_comment(raw));
    size_t ind = 0;
    while (ind < s.size() && s[ind] == ' ') ++ind;
    if (ind == s.size()) {
      if (p > text.size()) break;
      continue;
    }
    if (s[ind] == '\t') perr("line " + std::to_string(no) + ": tab in indentation");
    const std::string body = s.substr(ind);
    if (ind == 0 && (body == "---" || body.rfind("--- ", 0) == 0)) {
      if (started) perr("line " + std::to_string(no) + ": more than one document");
      if (body != "---") perr("line " + std::to_string(no) + ": content after the document marker");
      started = true;
      continue;
    }
    if (ind == 0 && body == "...") break;
    if (body[0] == '%') perr("line " + std::to_string(no) + ": directives are not supported");
    started = true;
    if (!out.empty() && bracket_depth(out.back().text) > 0) {
      out.back().text += "\n" + body;  // a flow collection continued on this line
    } else {
      out.push_back({(int)ind, body, no});
    }
    if (p > text.size()) break;
  }
  if (!out.empty() && bracket_depth(out.back().text) != 0) perr("unbalanced brackets in a flow collection");
  return out;
}

std::string where(const Line& l) { return "line " + std::to_string(l.no) + ": "; }

void unsupported(const std::string& s, const std::string& at) {
  if (!s.empty() && std::strchr("&*!|>%@`", s[0])) perr(at + "unsupported YAML form `" + s.substr(0, 12) + "`");
}

// a quoted scalar starting at s[i]; returns its value and moves i past it
std::string quoted(const std::string& s, size_t& i, const std::string& at) {
  const char q = s[i++];
  std::string v;
  while (i < s.size()) {
    const char c = s[i];
    if (q == '\'') {
      if (c == '\'') {
        if (i + 1 < s.size() && s[i + 1] == '\'') { v += '\''; i += 2; continue; }
        ++i;
        return v;
      }
      v += c;
      ++i;
    } else {
      if (c == '"') { ++i; return v; }
      if (c == '\\') {
        if (i + 1 >= s.size()) break;
        const char e = s[i + 1];
        switch (e) {
          case 'n': v += '\n'; break;
          case 't': v += '\t'; break;
          case '\\': v += '\\'; break;
          case '"': v += '"'; break;
          case '/': v += '/'; break;
          case '0': v += '\0'; break;
          default: perr(at + "unsupported escape in a double-quoted scalar");
        }
        i += 2;
        continue;
      }
      v += c;
      ++i;
    }
  }
  perr(at + "unterminated quoted scalar");
}

Node flow(const std::string& s, size_t& i, const std::string& at);

void skip_ws(const std::string& s, size_t& i) {
  while (i < s.size() && (s[i] == ' ' || s[i] == '\t' || s[i] == '\n')) ++i;
}

// one element of a flow collection (a nested collection, a quoted scalar or a
// plain scalar ending at , ] or })
Node flow_item(const std::string& s, size_t& i, const std::string& at) {
  skip_ws(s, i);
  Node n;
  if (i < s.size() && (s[i] == '[' || s[i] == '{')) return flow(s, i, at);
  if (i < s.size() && (s[i] == '"' || s[i] == '\'')) {
    n.kind = Node::kScalar;
    n.plain = false;
    n.text = quoted(s, i, at);
    return n;
  }
  size_t j = i;  // a plain scalar in a flow collection ends at a flow indicator
  while (j < s.size() && !std::strchr(",[]{}", s[j])) ++j;
  std::string t;
  for (char c : trim(s.substr(i, j - i))) {  // a line break inside a plain scalar folds to one blank
    if (c == '\n') {
      while (!t.empty() && t.back() == ' ') t.pop_back();
      t += ' ';
    } else {
      t += c;
    }
  }
  i = j;
  unsupported(t, at);
  if (t.find(": ") != std::string::npos) perr(at + "a mapping inside a flow sequence is not supported");
  n.kind = Node::kScalar;
  n.text = t;
  return n;
}

Node flow(const std::string& s, size_t& i, const std::string& at) {
  Node n;
  const char open = s[i++];
  const char close = open == '[' ? ']' : '}';
  n.kind = open == '[' ? Node::kSeq : Node::kMap;
  while (true) {
    skip_ws(s, i);
    if (i >= s.size()) perr(at + "unterminated flow collection");
    if (s[i] == close) { ++i; return n; }
    if (open == '[') {
      n.items.push_back(flow_item(s, i, at));
    } else {
      std::string key;
      if (s[i] == '"' || s[i] == '\'') {
        key = quoted(s, i, at);
      } else {
        // a plain key ends at a `:` followed by a blank, a flow indicator
        // (`,` `[` `]` `{` `}`) or the end (a `:` before anything else is part
        // of the scalar), or at `,` / `}`
        size_t j = i;
        while (j < s.size() && s[j] != ',' && s[j] != '}' &&
               !(s[j] == ':' && (j + 1 == s.size() || std::strchr(" \n,[]{}", s[j + 1]) != nullptr)))
          ++j;
        const std::string raw_key = s.substr(i, j - i);
        if (raw_key.find('\n') != std::string::npos) perr(at + "a mapping key spans lines");
        key = trim(raw_key);
        if (!key.empty() && (key[0] == '[' || key[0] == '{')) perr(at + "a collection as a mapping key");
        unsupported(key, at);
        i = j;
      }
      skip_ws(s, i);
      Node v;
      if (i < s.size() && s[i] == ':') {
        ++i;
        skip_ws(s, i);
        if (i < s.size() && s[i] != ',' && s[i] != '}') v = flow_item(s, i, at);
      }
      for (auto& e : n.entries)
        if (e.first == key) perr(at + "duplicate field `" + key + "`");
      n.entries.emplace_back(key, std::move(v));
    }
    skip_ws(s, i);
    if (i < s.size() && s[i] == ',') { ++i; continue; }
    if (i < s.size() && s[i] == close) { ++i; return n; }
    perr(at + "expected , or " + std::string(1, close) + " in a flow collection");
  }
}

// a value written after `key:` or `- ` on one line
Node inline_value(const std::string& v, const std::string& at) {
  Node n;
  if (v.empty()) return n;
  unsupported(v, at);
  size_t i = 0;
  if (v[0] == '[' || v[0] == '{') {
    n = flow(v, i, at);
  } else if (v[0] == '"' || v[0] == '\'') {
    n.kind = Node::kScalar;
    n.plain = false;
    n.text = quoted(v, i, at);
  } else {
    if (v.find(": ") != std::string::npos) perr(at + "mapping values are not allowed here");
    n.kind = Node::kScalar;
    n.text = v;
    return n;
  }
  skip_ws(v, i);
  if (i != v.size()) perr(at + "unexpected text after a value");
  return n;
}

bool is_dash(const std::string& t) { return t == "-" || t.rfind("- ", 0) == 0; }

// position of the `:` that ends a mapping key on this line, or npos
size_t key_colon(const std::string& t) {
  size_t i = 0;
  if (!t.empty() && (t[0] == '"' || t[0] == '\'')) {
    const char q = t[0];
    i = 1;
    while (i < t.size() && t[i] != q) ++i;
    ++i;
  }
  for (; i < t.size(); ++i) {
    if (t[i] == ':' && (i + 1 == t.size() || t[i + 1] == ' ')) return i;
    if (t[i] == '[' || t[i] == '{') return std::string::npos;
  }
  return std::string::npos;
}

struct Reader {
  std::vector<Line> lines;
  size_t i = 0;

  Node node(int indent) {
    if (i >= lines.size() || lines[i].indent < indent) return Node();
    const std::string& t = lines[i].text;
    if (is_dash(t)) return seq(lines[i].indent);
    if (t[0] == '[' || t[0] == '{' || key_colon(t) == std::string::npos) {
      // a flow collection or a scalar on a line of its own
      Node n = inline_value(t, where(lines[i]));
      ++i;
      return n;
    }
    return map(lines[i].indent);
  }

  Node seq(int ind) {
    Node n;
    n.kind = Node::kSeq;
    while (i < lines.size() && lines[i].indent == ind && is_dash(lines[i].text)) {
      Line& l = lines[i];
      size_t off = 1;
      while (off < l.text.size() && l.text[off] == ' ') ++off;
      const std::string rest = l.text.substr(off);
      if (rest.empty()) {
        ++i;
        n.items.push_back(i < lines.size() && lines[i].indent > ind ? node(lines[i].indent) : Node());
      } else if (rest[0] != '[' && rest[0] != '{' && rest[0] != '"' && rest[0] != '\'' &&
                 key_colon(rest) != std::string::npos) {
        // a mapping that starts on the dash line: its keys sit at the column of `rest`
        l.indent = ind + (int)off;
        l.text = rest;
        n.items.push_back(map(l.indent));
      } else {
        n.items.push_back(inline_value(rest, where(l)));
        ++i;
      }
    }
    if (i < lines.size() && lines[i].indent > ind) perr(where(lines[i]) + "bad indentation of a sequence entry");
    return n;
  }

  Node map(int ind) {
    Node n;
    n.kind = Node::kMap;
    while (i < lines.size() && lines[i].indent == ind && !is_dash(lines[i].text)) {
      const Line l = lines[i];
      const size_t c = key_colon(l.text);
      if (c == std::string::npos) perr(where(l) + "expected `key: value`");
      std::string key = trim(l.text.substr(0, c));
      if (!key.empty() && (key[0] == '"' || key[0] == '\'')) {
        size_t k = 0;
        key = quoted(key, k, where(l));
      } else {
        unsupported(key, where(l));
      }
      const std::string val = trim(l.text.substr(c + 1));
      ++i;
      Node v;
      if (val.empty()) {
        if (i < lines.size() && lines[i].indent > ind) v = node(lines[i].indent);
        else if (i < lines.size() && lines[i].indent == ind && is_dash(lines[i].text)) v = seq(ind);
      } else {
        v = inline_value(val, where(l));
      }
      for (auto& e : n.entries)
        if (e.first == key) perr(where(l) + "duplicate field `" + key + "`");
      n.entries.emplace_back(key, std::move(v));
    }
    if (i < lines.size() && lines[i].indent > ind) perr(where(lines[i]) + "bad indentation of a mapping entry");
    return n;
  }
};

Node read_yaml(const std::string& text) {
  Reader r;
  r.lines = split_lines(text);
  if (r.lines.empty()) return Node();
  Node root = r.node(r.lines[0].indent);
  if (r.i != r.lines.size()) perr(where(r.lines[r.i]) + "unexpected content");
  return root;
}

// ---------------------------------------------------------------------------
// The schema (settings.rs:27-454, as pwgpu/deck.py checks it)
// ---------------------------------------------------------------------------

const char* kElements =
    "H He Li Be B C N O F Ne Na Mg Al Si P S Cl Ar K Ca Sc Ti V Cr Mn Fe Co Ni Cu Zn Ga Ge As Se Br Kr "
    "Rb Sr Y Zr Nb Mo Tc Ru Rh Pd Ag Cd In Sn Sb Te I Xe Cs Ba La Ce Pr Nd Pm Sm Eu Gd Tb Dy Ho Er Tm "
    "Yb Lu Hf Ta W Re Os Ir Pt Au Hg Tl Pb Bi Po At Rn Fr Ra Ac Th Pa U Np Pu Am Cm Bk Cf Es Fm Md No "
    "Lr Rf Db Sg Bh Hs Mt Ds Rg Cn Nh Fl Mc Lv Ts Og";

bool is_element(const std::string& s) {
  if (s.empty() || s.find(' ') != std::string::npos) return false;
  const std::string hay = std::string(" ") + kElements + " ";
  return hay.find(" " + s + " ") != std::string::npos;
}

const Node* block(const Node* n, const std::string& at, std::initializer_list<const char*> fields) {
  static const Node empty = [] { Node e; e.kind = Node::kMap; return e; }();
  if (!n || n->kind == Node::kNull || (n->kind == Node::kScalar && n->plain && typed(n).type == Value::kNone))
    return &empty;
  if (n->kind != Node::kMap) perr(at + ": expected a mapping");
  for (auto& e : n->entries) {
    bool ok = false;
    for (const char* f : fields) ok |= e.first == f;
    if (!ok) {
      std::string list;
      for (const char* f : fields) list += (list.empty() ? "" : ", ") + std::string(f);
      perr(at + ": unknown field `" + e.first + "`, expected one of " + list);
    }
  }
  return n;
}

double num(const Node* n, const std::string& at) {
  const Value v = typed(n);
  if (v.type == Value::kInt) return (double)v.i;
  if (v.type == Value::kFloat) return v.f;
  perr(at + ": expected a number");
}
double num_or(const Node* n, double def, const std::string& at) { return n ? num(n, at) : def; }

int uint_(const Node* n, const std::string& at) {
  const Value v = typed(n);
  if (v.type != Value::kInt || v.i < 0 || v.i > INT32_MAX) perr(at + ": expected a non-negative integer");
  return (int)v.i;
}
int uint_or(const Node* n, int def, const std::string& at) { return n ? uint_(n, at) : def; }

int bool_(const Node* n, const std::string& at) {
  const Value v = typed(n);
  if (v.type != Value::kBool) perr(at + ": expected true or false");
  return v.b ? 1 : 0;
}
int bool_or(const Node* n, int def, const std::string& at) { return n ? bool_(n, at) : def; }

int choice(const Node* n, const std::string& def, const std::string& at, std::initializer_list<const char*> opts) {
  std::string s = def;
  if (n) {
    const Value v = typed(n);
    if (v.type != Value::kStr) perr(at + ": unknown variant");
    s = v.s;
  }
  int k = 0;
  for (const char* o : opts) {
    if (s == o) return k;
    ++k;
  }
  perr(at + ": unknown variant `" + s + "`");
}

template <typename F>
void vec3(const Node* n, const std::string& at, F conv) {
  if (!n || n->kind != Node::kSeq || n->items.size() != 3) perr(at + ": expected a list of 3 values");
  for (int k = 0; k < 3; ++k) conv(k, &n->items[k]);
}

// Python truthiness of an optional list-valued field (`value or []`)
bool empty_like(const Node* n) {
  if (!n || n->kind == Node::kNull) return true;
  if (n->kind == Node::kSeq) return n->items.empty();
  if (n->kind == Node::kMap) return n->entries.empty();
  const Value v = typed(n);
  return v.type == Value::kNone || (v.type == Value::kBool && !v.b) || (v.type == Value::kInt && v.i == 0) ||
         (v.type == Value::kFloat && v.f == 0.0) || (v.type == Value::kStr && v.s.empty());
}

std::string label_text(const Node* n) {
  const Value v = typed(n);
  switch (v.type) {
    case Value::kNone: return "None";
    case Value::kBool: return v.b ? "True" : "False";
    case Value::kInt: return std::to_string(v.i);
    case Value::kFloat: {
      char buf[64];
      auto r = std::to_chars(buf, buf + sizeof(buf), v.f);
      std::string s(buf, r.ptr);
      if (s.find_first_of(".eni") == std::string::npos) s += ".0";
      return s;
    }
    default: return v.s;
  }
}

}  // namespace

struct pwgpu_deck {
  pwgpu_deck_settings s{};
  std::vector<std::string> atom_symbols;
  std::vector<double> atom_pos;
  std::vector<std::string> mag_symbols;
  std::vector<double> mag_values;
  std::vector<std::string> path_labels;
  std::vector<double> path_frac;
};

namespace {

pwgpu_deck* build(const std::string& text) {
  const Node root = read_yaml(text);
  auto* d = new pwgpu_deck();
  try {
    pwgpu_deck_settings& s = d->s;
    const Node* top = block(&root, "settings", {"system", "basis", "kpoints", "scf", "electrons", "xc", "symmetry",
                                                 "output", "initial_density"});
    for (const char* req : {"system", "kpoints"})
      if (!top->get(req)) perr(std::string("missing field `") + req + "`");
    const Node* sys = block(top->get("system"), "system", {"lattice", "atoms"});
    const Node* lat = sys->get("lattice");
    if (!lat) perr("system: missing field `lattice`");
    if (lat->kind != Node::kSeq || lat->items.size() != 3) perr("system.lattice: expected 3 vectors");
    for (int r = 0; r < 3; ++r)
      vec3(&lat->items[r], "system.lattice", [&](int k, const Node* x) { s.lattice[3 * r + k] = num(x, "system.lattice"); });
    const Node* atoms = sys->get("atoms");
    if (!empty_like(atoms)) {
      if (atoms->kind != Node::kSeq) perr("system.atoms: expected a list");
      for (size_t a = 0; a < atoms->items.size(); ++a) {
        const std::string at = "system.atoms[" + std::to_string(a) + "]";
        const Node* ab = block(&atoms->items[a], at, {"symbol", "position"});
        for (const char* req : {"symbol", "position"})
          if (!ab->get(req)) perr(at + ": missing field `" + req + "`");
        const Value sym = typed(ab->get("symbol"));
        if (sym.type != Value::kStr || !is_element(sym.s)) perr(at + ".symbol: unknown element");
        d->atom_symbols.push_back(sym.s);
        vec3(ab->get("position"), at + ".position",
             [&](int, const Node* x) { d->atom_pos.push_back(num(x, at + ".position")); });
      }
    }
    s.n_atoms = (int32_t)d->atom_symbols.size();

    const Node* bb = block(top->get("basis"), "basis", {"ecutwfc", "ecutrho_ratio", "fft_grid"});
    s.ecutwfc = num_or(bb->get("ecutwfc"), 300.0, "basis.ecutwfc");
    s.ecutrho_ratio = uint_or(bb->get("ecutrho_ratio"), 4, "basis.ecutrho_ratio");
    const Node* fg = bb->get("fft_grid");
    if (fg && typed(fg).type != Value::kNone)
      vec3(fg, "basis.fft_grid", [&](int k, const Node* x) { s.fft_grid[k] = uint_(x, "basis.fft_grid"); });

    const Node* kb = top->get("kpoints");
    if (kb->kind != Node::kMap || !kb->get("type")) perr("kpoints: missing field `type`");
    s.kpoints_type = choice(kb->get("type"), "", "kpoints.type", {"monkhorst_pack", "band_path"});
    if (s.kpoints_type == PWGPU_KPOINTS_MONKHORST_PACK) {
      kb = block(kb, "kpoints", {"type", "grid", "shift"});
      if (!kb->get("grid")) perr("kpoints: missing field `grid`");
      const Node* sh = kb->get("shift");
      if (sh && sh->kind == Node::kMap) {
        const Node* sb = block(sh, "kpoints.shift", {"custom"});
        vec3(sb->get("custom"), "kpoints.shift.custom",
             [&](int k, const Node* x) { s.mp_shift[k] = uint_(x, "kpoints.shift.custom"); });
        for (int k = 0; k < 3; ++k)
          if (s.mp_shift[k] > 1) throw InvalidParam{"kpoints.shift.custom: half-shift flags must be 0 or 1"};
      } else {
        const int c = choice(sh, "gamma_centered", "kpoints.shift", {"gamma_centered", "mp1976", "mp_1976", "shifted"});
        for (int k = 0; k < 3; ++k) s.mp_shift[k] = c == 0 ? 0 : 1;
      }
      vec3(kb->get("grid"), "kpoints.grid", [&](int k, const Node* x) { s.mp_grid[k] = uint_(x, "kpoints.grid"); });
    } else {
      kb = block(kb, "kpoints", {"type", "path", "npoints"});
      const Node* path = kb->get("path");
      if (!empty_like(path)) {
        if (path->kind != Node::kSeq) perr("kpoints.path: expected a list");
        for (size_t p = 0; p < path->items.size(); ++p) {
          const std::string at = "kpoints.path[" + std::to_string(p) + "]";
          const Node* pb = block(&path->items[p], at, {"label", "frac"});
          d->path_labels.push_back(label_text(pb->get("label")));
          vec3(pb->get("frac"), at + ".frac", [&](int, const Node* x) { d->path_frac.push_back(num(x, at + ".frac")); });
        }
      }
      s.n_path = (int32_t)d->path_labels.size();
      s.band_npoints = uint_or(kb->get("npoints"), 50, "kpoints.npoints");
    }

    const Node* sb = block(top->get("scf"), "scf",
                           {"max_iter", "conv_threshold", "energy_threshold", "n_bands", "eigensolver", "wfrx_subspace",
                            "mixing_beta", "mixing_ndim", "mixing_mode", "pulay_period", "adaptive_beta", "smearing",
                            "smearing_width"});
    s.max_iter = uint_or(sb->get("max_iter"), 50, "scf.max_iter");
    s.conv_threshold = num_or(sb->get("conv_threshold"), 1e-6, "scf.conv_threshold");
    s.energy_threshold = num_or(sb->get("energy_threshold"), 1e-5, "scf.energy_threshold");
    const Node* nb = sb->get("n_bands");
    s.n_bands = (!nb || typed(nb).type == Value::kNone) ? -1 : uint_(nb, "scf.n_bands");
    s.eigensolver = choice(sb->get("eigensolver"), "dense", "scf.eigensolver", {"dense", "iterative"});
    s.wfrx_subspace = bool_or(sb->get("wfrx_subspace"), 0, "scf.wfrx_subspace");
    s.mixing_beta = num_or(sb->get("mixing_beta"), 0.3, "scf.mixing_beta");
    s.mixing_ndim = uint_or(sb->get("mixing_ndim"), 8, "scf.mixing_ndim");
    s.mixing_mode = choice(sb->get("mixing_mode"), "plain", "scf.mixing_mode",
                           {"plain", "kerker", "broyden", "broyden_kerker", "periodic_pulay", "periodic_pulay_kerker"});
    s.pulay_period = uint_or(sb->get("pulay_period"), 3, "scf.pulay_period");
    s.adaptive_beta = bool_or(sb->get("adaptive_beta"), 0, "scf.adaptive_beta");
    s.smearing = choice(sb->get("smearing"), "fermi_dirac", "scf.smearing",
                        {"fermi_dirac", "gaussian", "methfessel_paxton", "cold", "fixed"});
    s.smearing_width = num_or(sb->get("smearing_width"), 0.05, "scf.smearing_width");

    const Node* eb = block(top->get("electrons"), "electrons",
                           {"spin_polarized", "starting_magnetization", "tot_magnetization", "occupations"});
    const Node* sm = eb->get("starting_magnetization");
    if (!empty_like(sm)) {
      if (sm->kind != Node::kMap) perr("electrons.starting_magnetization: expected a mapping");
      for (auto& e : sm->entries) {
        Node key;
        key.kind = Node::kScalar;
        key.text = e.first;
        const Value kv = typed(&key);
        if (kv.type != Value::kStr || !is_element(kv.s)) perr("electrons.starting_magnetization: unknown element");
        d->mag_symbols.push_back(kv.s);
        d->mag_values.push_back(num(&e.second, "electrons.starting_magnetization." + e.first));
      }
    }
    s.n_starting_magnetization = (int32_t)d->mag_symbols.size();
    s.spin_polarized = bool_or(eb->get("spin_polarized"), 0, "electrons.spin_polarized");
    const Node* tm = eb->get("tot_magnetization");
    if (tm && typed(tm).type != Value::kNone) {
      s.has_tot_magnetization = 1;
      s.tot_magnetization = num(tm, "electrons.tot_magnetization");
    }
    s.occupations = choice(eb->get("occupations"), "smearing", "electrons.occupations", {"smearing", "fixed"});

    const Node* xb = block(top->get("xc"), "xc", {"functional"});
    s.functional = choice(xb->get("functional"), "pz", "xc.functional", {"pz", "pbe", "pbe0", "hse06"});
    const Node* yb = block(top->get("symmetry"), "symmetry", {"enabled", "time_reversal", "tolerance"});
    s.symmetry_enabled = bool_or(yb->get("enabled"), 1, "symmetry.enabled");
    s.time_reversal = bool_or(yb->get("time_reversal"), 1, "symmetry.time_reversal");
    s.symmetry_tolerance = num_or(yb->get("tolerance"), 1e-5, "symmetry.tolerance");
    const Node* ob = block(top->get("output"), "output", {"verbosity", "write_density", "write_bands"});
    s.verbosity = choice(ob->get("verbosity"), "normal", "output.verbosity", {"low", "normal", "high"});
    s.write_density = bool_or(ob->get("write_density"), 0, "output.write_density");
    s.write_bands = bool_or(ob->get("write_bands"), 1, "output.write_bands");
    const Node* ib = block(top->get("initial_density"), "initial_density", {"gaussian_sigma"});
    s.gaussian_sigma = num_or(ib->get("gaussian_sigma"), 1.0, "initial_density.gaussian_sigma");
  } catch (...) {
    delete d;
    throw;
  }
  return d;
}

void copy_names(const std::vector<std::string>& names, char* out, size_t width) {
  for (size_t k = 0; k < names.size(); ++k) std::snprintf(out + k * width, width, "%s", names[k].c_str());
}

}  // namespace

extern "C" {

pwgpu_status pwgpu_deck_parse(const char* text, int64_t len, pwgpu_deck** out) {
  if (!text || !out || len < 0) return fail(PWGPU_E_INVALID, "pwgpu_deck_parse: NULL argument or negative length");
  *out = nullptr;
  try {
    *out = build(std::string(text, (size_t)len));
  } catch (const ParseError& e) {
    return fail(PWGPU_E_PARSE, "YAML parse error: " + e.msg);
  } catch (const InvalidParam& e) {
    return fail(PWGPU_E_INVALID, e.msg);
  } catch (const std::bad_alloc&) {
    return fail(PWGPU_E_OOM, "pwgpu_deck_parse: out of host memory");
  }
  return PWGPU_OK;
}

pwgpu_status pwgpu_deck_get_settings(const pwgpu_deck* d, pwgpu_deck_settings* s) {
  if (!d || !s) return fail(PWGPU_E_INVALID, "pwgpu_deck_get_settings: NULL argument");
  *s = d->s;
  return PWGPU_OK;
}

pwgpu_status pwgpu_deck_get_atoms(const pwgpu_deck* d, char* symbols, double* positions) {
  if (!d || !symbols || !positions) return fail(PWGPU_E_INVALID, "pwgpu_deck_get_atoms: NULL argument");
  copy_names(d->atom_symbols, symbols, 8);
  if (!d->atom_pos.empty()) std::memcpy(positions, d->atom_pos.data(), d->atom_pos.size() * sizeof(double));
  return PWGPU_OK;
}

pwgpu_status pwgpu_deck_get_starting_magnetization(const pwgpu_deck* d, char* symbols, double* values) {
  if (!d || !symbols || !values) return fail(PWGPU_E_INVALID, "pwgpu_deck_get_starting_magnetization: NULL argument");
  copy_names(d->mag_symbols, symbols, 8);
  if (!d->mag_values.empty()) std::memcpy(values, d->mag_values.data(), d->mag_values.size() * sizeof(double));
  return PWGPU_OK;
}

pwgpu_status pwgpu_deck_get_band_path(const pwgpu_deck* d, char* labels, double* frac) {
  if (!d || !labels || !frac) return fail(PWGPU_E_INVALID, "pwgpu_deck_get_band_path: NULL argument");
  copy_names(d->path_labels, labels, 16);
  if (!d->path_frac.empty()) std::memcpy(frac, d->path_frac.data(), d->path_frac.size() * sizeof(double));
  return PWGPU_OK;
}

pwgpu_status pwgpu_deck_free(pwgpu_deck* d) {
  delete d;
  return PWGPU_OK;
}

}  // extern "C"
