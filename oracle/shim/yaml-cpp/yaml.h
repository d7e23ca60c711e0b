// Minimal YAML reader exposing the small part of the yaml-cpp API that the
// reference's input-deck parser uses (LoadFile, operator[], operator bool,
// as<T>(), size(), iteration over sequences and maps).
//
// ORACLE TEST INFRASTRUCTURE ONLY: this header lets the reference's own
// src/inp/input.cpp be compiled unchanged inside this container, where
// yaml-cpp is not installed.  It is never linked into the product library.
//
// Supported subset (what the reference's example decks use): block mappings
// by indentation, block sequences ("- item"), flow sequences ("[a, b]",
// nested), plain / single- / double-quoted scalars, "#" comments.
#pragma once

#include <cstdlib>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace YAML {

namespace detail {

struct Data {
  enum Kind { Null, Scalar, Sequence, Map } kind = Null;
  std::string scalar;
  std::vector<std::shared_ptr<Data>> seq;
  std::vector<std::pair<std::string, std::shared_ptr<Data>>> map;
};

inline std::string trim(const std::string &s) {
  size_t a = s.find_first_not_of(" \t\r\n");
  if (a == std::string::npos) return "";
  size_t b = s.find_last_not_of(" \t\r\n");
  return s.substr(a, b - a + 1);
}

inline std::string unquote(const std::string &s0) {
  std::string s = trim(s0);
  if (s.size() >= 2 && ((s.front() == '"' && s.back() == '"') ||
                        (s.front() == '\'' && s.back() == '\'')))
    return s.substr(1, s.size() - 2);
  return s;
}

// strip a trailing comment that is not inside quotes
inline std::string stripComment(const std::string &line) {
  bool sq = false, dq = false;
  for (size_t i = 0; i < line.size(); i++) {
    char c = line[i];
    if (c == '\'' && !dq) sq = !sq;
    else if (c == '"' && !sq) dq = !dq;
    else if (c == '#' && !sq && !dq && (i == 0 || line[i - 1] == ' ' || line[i - 1] == '\t'))
      return line.substr(0, i);
  }
  return line;
}

// parse a flow collection "[...]" or a scalar
inline std::shared_ptr<Data> parseFlow(const std::string &text, size_t &pos);

inline void skipWs(const std::string &t, size_t &p) {
  while (p < t.size() && (t[p] == ' ' || t[p] == '\t')) p++;
}

inline std::shared_ptr<Data> parseFlow(const std::string &t, size_t &p) {
  skipWs(t, p);
  auto d = std::make_shared<Data>();
  if (p < t.size() && t[p] == '[') {
    d->kind = Data::Sequence;
    p++;
    skipWs(t, p);
    if (p < t.size() && t[p] == ']') { p++; return d; }
    while (p < t.size()) {
      d->seq.push_back(parseFlow(t, p));
      skipWs(t, p);
      if (p < t.size() && t[p] == ',') { p++; continue; }
      if (p < t.size() && t[p] == ']') { p++; break; }
      throw std::runtime_error("yaml shim: malformed flow sequence: " + t);
    }
    return d;
  }
  size_t start = p;
  if (p < t.size() && (t[p] == '"' || t[p] == '\'')) {
    char q = t[p++];
    while (p < t.size() && t[p] != q) p++;
    p++;
  } else {
    while (p < t.size() && t[p] != ',' && t[p] != ']') p++;
  }
  d->kind = Data::Scalar;
  d->scalar = unquote(t.substr(start, p - start));
  return d;
}

struct Line {
  int indent;
  std::string text;  // content without indentation / comments
};

class Parser {
public:
  explicit Parser(std::vector<Line> lines) : L(std::move(lines)) {}

  std::shared_ptr<Data> parseDocument() {
    size_t i = 0;
    if (L.empty()) return std::make_shared<Data>();
    return parseBlock(i, L[0].indent);
  }

private:
  std::vector<Line> L;

  static bool isSeqItem(const std::string &t) {
    return t == "-" || (t.size() >= 2 && t[0] == '-' && t[1] == ' ');
  }

  // position of the "key: " separator, or npos
  static size_t keySep(const std::string &t) {
    bool sq = false, dq = false;
    int depth = 0;
    for (size_t k = 0; k < t.size(); k++) {
      char c = t[k];
      if (c == '\'' && !dq) sq = !sq;
      else if (c == '"' && !sq) dq = !dq;
      else if (!sq && !dq) {
        if (c == '[' || c == '{') depth++;
        else if (c == ']' || c == '}') depth--;
        else if (c == ':' && depth == 0 && (k + 1 == t.size() || t[k + 1] == ' ' || t[k + 1] == '\t'))
          return k;
      }
    }
    return std::string::npos;
  }

  std::shared_ptr<Data> parseValueText(const std::string &v) {
    size_t p = 0;
    return parseFlow(v, p);
  }

  std::shared_ptr<Data> parseBlock(size_t &i, int indent) {
    if (isSeqItem(L[i].text)) return parseSeq(i, indent);
    return parseMap(i, indent);
  }

  std::shared_ptr<Data> parseSeq(size_t &i, int indent) {
    auto d = std::make_shared<Data>();
    d->kind = Data::Sequence;
    while (i < L.size() && L[i].indent == indent && isSeqItem(L[i].text)) {
      std::string rest = trim(L[i].text.substr(1));
      if (rest.empty()) {
        i++;
        if (i < L.size() && L[i].indent > indent) d->seq.push_back(parseBlock(i, L[i].indent));
        else d->seq.push_back(std::make_shared<Data>());
      } else if (keySep(rest) != std::string::npos) {
        // "- key: value" opens a mapping whose further keys are indented
        int item_indent = indent + 2;
        L[i].indent = item_indent;
        L[i].text = rest;
        d->seq.push_back(parseMap(i, item_indent));
      } else {
        d->seq.push_back(parseValueText(rest));
        i++;
      }
    }
    return d;
  }

  std::shared_ptr<Data> parseMap(size_t &i, int indent) {
    auto d = std::make_shared<Data>();
    d->kind = Data::Map;
    while (i < L.size() && L[i].indent == indent && !isSeqItem(L[i].text)) {
      const std::string &t = L[i].text;
      size_t c = keySep(t);
      if (c == std::string::npos)
        throw std::runtime_error("yaml shim: expected 'key: value' in line: " + t);
      std::string key = unquote(t.substr(0, c));
      std::string val = trim(t.substr(c + 1));
      i++;
      std::shared_ptr<Data> child;
      if (!val.empty()) {
        child = parseValueText(val);
      } else if (i < L.size() && (L[i].indent > indent ||
                                  (L[i].indent == indent && isSeqItem(L[i].text)))) {
        child = parseBlock(i, L[i].indent);
      } else {
        child = std::make_shared<Data>();  // null value
      }
      d->map.emplace_back(key, child);
    }
    return d;
  }
};

inline std::shared_ptr<Data> parseText(const std::string &text) {
  std::vector<Line> lines;
  std::istringstream is(text);
  std::string raw;
  while (std::getline(is, raw)) {
    std::string s = stripComment(raw);
    if (trim(s).empty()) continue;
    if (trim(s) == "---") continue;
    int ind = 0;
    while (ind < (int)s.size() && s[ind] == ' ') ind++;
    lines.push_back({ind, trim(s)});
  }
  return Parser(std::move(lines)).parseDocument();
}

template <class T> struct convert;

template <> struct convert<std::string> {
  static std::string get(const std::string &s) { return s; }
};
template <> struct convert<double> {
  static double get(const std::string &s) {
    char *e = nullptr;
    double v = std::strtod(s.c_str(), &e);
    if (e == s.c_str()) throw std::runtime_error("yaml shim: bad double '" + s + "'");
    return v;
  }
};
template <> struct convert<float> {
  static float get(const std::string &s) { return (float)convert<double>::get(s); }
};
template <> struct convert<int> {
  static int get(const std::string &s) {
    char *e = nullptr;
    long v = std::strtol(s.c_str(), &e, 10);
    if (e == s.c_str()) throw std::runtime_error("yaml shim: bad int '" + s + "'");
    return (int)v;
  }
};
template <> struct convert<long> {
  static long get(const std::string &s) { return convert<int>::get(s); }
};
template <> struct convert<unsigned long> {
  static unsigned long get(const std::string &s) {
    char *e = nullptr;
    unsigned long v = std::strtoul(s.c_str(), &e, 10);
    if (e == s.c_str()) throw std::runtime_error("yaml shim: bad size_t '" + s + "'");
    return v;
  }
};
template <> struct convert<unsigned int> {
  static unsigned int get(const std::string &s) { return (unsigned int)convert<unsigned long>::get(s); }
};
template <> struct convert<bool> {
  static bool get(const std::string &s) {
    if (s == "true" || s == "True" || s == "TRUE" || s == "yes" || s == "on" || s == "1")
      return true;
    if (s == "false" || s == "False" || s == "FALSE" || s == "no" || s == "off" || s == "0")
      return false;
    throw std::runtime_error("yaml shim: bad bool '" + s + "'");
  }
};

}  // namespace detail

class Node {
public:
  Node() = default;
  explicit Node(std::shared_ptr<detail::Data> d) : d_(std::move(d)) {}

  bool IsDefined() const { return d_ != nullptr; }
  bool IsNull() const { return d_ && d_->kind == detail::Data::Null; }
  bool IsScalar() const { return d_ && d_->kind == detail::Data::Scalar; }
  bool IsSequence() const { return d_ && d_->kind == detail::Data::Sequence; }
  bool IsMap() const { return d_ && d_->kind == detail::Data::Map; }
  explicit operator bool() const { return IsDefined(); }
  bool operator!() const { return !IsDefined(); }

  Node operator[](const std::string &key) const {
    if (!d_ || d_->kind != detail::Data::Map) return Node();
    for (auto &kv : d_->map)
      if (kv.first == key) return Node(kv.second);
    return Node();
  }
  Node operator[](const char *key) const { return (*this)[std::string(key)]; }
  Node operator[](int idx) const { return at((size_t)idx); }
  Node operator[](size_t idx) const { return at(idx); }

  size_t size() const {
    if (!d_) return 0;
    if (d_->kind == detail::Data::Sequence) return d_->seq.size();
    if (d_->kind == detail::Data::Map) return d_->map.size();
    return 0;
  }

  template <class T> T as() const {
    if (!d_) throw std::runtime_error("yaml shim: as<>() on undefined node");
    if (d_->kind != detail::Data::Scalar)
      throw std::runtime_error("yaml shim: as<>() on non-scalar node");
    return detail::convert<T>::get(d_->scalar);
  }

  const std::string &Scalar() const {
    static const std::string empty;
    return d_ && d_->kind == detail::Data::Scalar ? d_->scalar : empty;
  }

  class const_iterator;
  using iterator = const_iterator;

  const_iterator begin() const;
  const_iterator end() const;

private:
  Node at(size_t idx) const {
    if (!d_ || d_->kind != detail::Data::Sequence || idx >= d_->seq.size()) return Node();
    return Node(d_->seq[idx]);
  }
  std::shared_ptr<detail::Data> d_;
};

// iteration: sequences yield nodes; maps yield key/value pairs exposed as
// first/second (both Nodes), like yaml-cpp's iterator value.
struct iterator_value : public Node {
  Node first, second;
  iterator_value() = default;
  explicit iterator_value(const Node &n) : Node(n) {}
  iterator_value(const Node &k, const Node &v) : first(k), second(v) {}
};

class Node::const_iterator {
public:
  const_iterator(const detail::Data *d, size_t i) : d_(d), i_(i) {}
  bool operator!=(const const_iterator &o) const { return i_ != o.i_ || d_ != o.d_; }
  bool operator==(const const_iterator &o) const { return !(*this != o); }
  const_iterator &operator++() { ++i_; return *this; }
  iterator_value operator*() const {
    if (d_->kind == detail::Data::Sequence) return iterator_value(Node(d_->seq[i_]));
    auto k = std::make_shared<detail::Data>();
    k->kind = detail::Data::Scalar;
    k->scalar = d_->map[i_].first;
    return iterator_value(Node(k), Node(d_->map[i_].second));
  }
  struct arrow_proxy {
    iterator_value v;
    const iterator_value *operator->() const { return &v; }
  };
  arrow_proxy operator->() const { return {**this}; }

private:
  const detail::Data *d_;
  size_t i_;
};

inline Node::const_iterator Node::begin() const { return const_iterator(d_.get(), 0); }
inline Node::const_iterator Node::end() const { return const_iterator(d_.get(), size()); }

inline Node Load(const std::string &text) { return Node(detail::parseText(text)); }

inline Node LoadFile(const std::string &filename) {
  std::ifstream f(filename);
  if (!f) throw std::runtime_error("yaml shim: cannot open file " + filename);
  std::stringstream ss;
  ss << f.rdbuf();
  return Load(ss.str());
}

}  // namespace YAML
