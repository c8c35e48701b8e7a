#include "xml.h"

#include <cctype>
#include <cstring>

namespace mjb {
namespace {

struct Reader {
  const std::string& s;
  size_t i = 0;
  int line = 1;

  [[noreturn]] void fail(const std::string& msg) const {
    throw std::runtime_error("XML parse error at line " + std::to_string(line) + ": " + msg);
  }
  bool eof() const { return i >= s.size(); }
  char peek() const { return eof() ? '\0' : s[i]; }
  void adv(size_t n = 1) {
    for (size_t k = 0; k < n && i < s.size(); k++, i++)
      if (s[i] == '\n') line++;
  }
  bool starts(const char* p) const { return s.compare(i, std::strlen(p), p) == 0; }
  void skip_ws() {
    while (!eof() && std::isspace(static_cast<unsigned char>(peek()))) adv();
  }
  void skip_until(const char* end) {
    size_t n = std::strlen(end);
    while (!eof() && !starts(end)) adv();
    if (eof()) fail(std::string("unterminated construct, expected '") + end + "'");
    adv(n);
  }
  // Skips whitespace, comments, processing instructions and doctype.
  void skip_misc() {
    for (;;) {
      skip_ws();
      if (starts("<!--")) skip_until("-->");
      else if (starts("<?")) skip_until("?>");
      else if (starts("<!")) skip_until(">");
      else return;
    }
  }
  std::string name() {
    size_t b = i;
    while (!eof() && (std::isalnum(static_cast<unsigned char>(peek())) || peek() == '_' || peek() == '-' || peek() == ':' || peek() == '.')) adv();
    if (b == i) fail("expected a name");
    return s.substr(b, i - b);
  }
  static std::string unescape(const std::string& v) {
    std::string out;
    for (size_t k = 0; k < v.size(); k++) {
      if (v[k] == '&') {
        size_t e = v.find(';', k);
        if (e != std::string::npos) {
          std::string ent = v.substr(k + 1, e - k - 1);
          if (ent == "lt") { out += '<'; k = e; continue; }
          if (ent == "gt") { out += '>'; k = e; continue; }
          if (ent == "amp") { out += '&'; k = e; continue; }
          if (ent == "quot") { out += '"'; k = e; continue; }
          if (ent == "apos") { out += '\''; k = e; continue; }
        }
      }
      out += v[k];
    }
    return out;
  }
  XmlNode element() {
    if (peek() != '<') fail("expected '<'");
    XmlNode n;
    n.line = line;
    adv();
    n.tag = name();
    for (;;) {
      skip_ws();
      if (starts("/>")) { adv(2); return n; }
      if (peek() == '>') { adv(); break; }
      std::string an = name();
      skip_ws();
      if (peek() != '=') fail("expected '=' after attribute " + an);
      adv();
      skip_ws();
      char q = peek();
      if (q != '"' && q != '\'') fail("expected quoted value for attribute " + an);
      adv();
      size_t b = i;
      while (!eof() && peek() != q) adv();
      if (eof()) fail("unterminated attribute value");
      n.attrs.emplace_back(an, unescape(s.substr(b, i - b)));
      adv();
    }
    // children and text (text content is ignored)
    for (;;) {
      skip_misc();
      if (eof()) fail("unterminated element <" + n.tag + ">");
      if (starts("</")) {
        adv(2);
        std::string en = name();
        if (en != n.tag) fail("mismatched closing tag </" + en + "> for <" + n.tag + ">");
        skip_ws();
        if (peek() != '>') fail("expected '>'");
        adv();
        return n;
      }
      if (peek() == '<') {
        n.children.push_back(element());
      } else {
        while (!eof() && peek() != '<') adv();
      }
    }
  }
};

}  // namespace

XmlNode parse_xml(const std::string& text) {
  Reader r{text};
  r.skip_misc();
  if (r.eof()) r.fail("empty document");
  XmlNode root = r.element();
  r.skip_misc();
  if (!r.eof()) r.fail("trailing content after root element");
  return root;
}

}  // namespace mjb
