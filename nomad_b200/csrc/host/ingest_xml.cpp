// A small XML reader for scene files: elements, attributes, comments, processing instructions,
// CDATA and DOCTYPE (the last three skipped), elements nested at most 500 deep. It accepts what the reference's vendored tinyxml2
// accepts for scene documents and reports mismatched or unclosed tags and malformed attributes.
// Attribute values get tinyxml2's treatment: the five predefined entities and numeric character
// references decoded (an unknown entity is kept as written), line endings normalised to "\n".
#include <cstring>

#include "ingest.h"

namespace nomad {
namespace ingest {

const char *XmlElem::attr(const char *n) const {
  for (const XmlAttr &a : attrs)
    if (a.name == n) return a.value.c_str();
  return nullptr;
}

namespace {

inline bool ws(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\v' || c == '\f'; }
inline bool name_start(unsigned char c) { return (c >= 'A' && c <= 'Z') || (c >= 'a' && c <= 'z') || c == '_' || c == ':' || c >= 0x80; }
inline bool name_char(unsigned char c) { return name_start(c) || (c >= '0' && c <= '9') || c == '-' || c == '.'; }

void put_utf8(std::string &o, unsigned long cp) {
  if (cp < 0x80) {
    o += static_cast<char>(cp);
  } else if (cp < 0x800) {
    o += static_cast<char>(0xC0 | (cp >> 6));
    o += static_cast<char>(0x80 | (cp & 0x3F));
  } else if (cp < 0x10000) {
    o += static_cast<char>(0xE0 | (cp >> 12));
    o += static_cast<char>(0x80 | ((cp >> 6) & 0x3F));
    o += static_cast<char>(0x80 | (cp & 0x3F));
  } else {
    o += static_cast<char>(0xF0 | (cp >> 18));
    o += static_cast<char>(0x80 | ((cp >> 12) & 0x3F));
    o += static_cast<char>(0x80 | ((cp >> 6) & 0x3F));
    o += static_cast<char>(0x80 | (cp & 0x3F));
  }
}

std::string decode(const char *s, size_t n) {
  std::string o;
  o.reserve(n);
  for (size_t i = 0; i < n; ++i) {
    const char c = s[i];
    if (c == '\r') {
      o += '\n';
      if (i + 1 < n && s[i + 1] == '\n') ++i;
      continue;
    }
    if (c != '&') {
      o += c;
      continue;
    }
    static const struct {
      const char *name;
      char ch;
    } kEnt[] = {{"quot;", '"'}, {"amp;", '&'}, {"apos;", '\''}, {"lt;", '<'}, {"gt;", '>'}};
    bool done = false;
    for (const auto &e : kEnt) {
      const size_t len = std::strlen(e.name);
      if (i + 1 + len <= n && std::strncmp(s + i + 1, e.name, len) == 0) {
        o += e.ch;
        i += len;
        done = true;
        break;
      }
    }
    if (done) continue;
    if (i + 2 < n && s[i + 1] == '#') {
      size_t j = i + 2;
      const bool hex = s[j] == 'x' || s[j] == 'X';
      if (hex) ++j;
      unsigned long cp = 0;
      size_t digits = 0;
      while (j < n && s[j] != ';') {
        const char d = s[j];
        int v = -1;
        if (d >= '0' && d <= '9') v = d - '0';
        else if (hex && d >= 'a' && d <= 'f') v = d - 'a' + 10;
        else if (hex && d >= 'A' && d <= 'F') v = d - 'A' + 10;
        if (v < 0 || cp > 0x10FFFF) break;
        cp = cp * (hex ? 16 : 10) + static_cast<unsigned long>(v);
        ++digits;
        ++j;
      }
      if (j < n && s[j] == ';' && digits > 0 && cp <= 0x10FFFF) {
        put_utf8(o, cp);
        i = j;
        continue;
      }
    }
    o += c;  // unknown entity: kept as written
  }
  return o;
}

// Deepest element nesting accepted (tinyxml2 rejects documents nested deeper than 500).
constexpr int kMaxDepth = 500;

struct Reader {
  const std::string &t;
  size_t p = 0;
  int depth = 0;
  std::string &err;
  Reader(const std::string &text, std::string &e) : t(text), err(e) {}

  bool fail(const char *what) {
    err = std::string(what) + " at byte " + std::to_string(p);
    return false;
  }
  bool starts(const char *s) const { return t.compare(p, std::strlen(s), s) == 0; }
  bool skip_past(const char *s) {
    const size_t q = t.find(s, p);
    if (q == std::string::npos) return false;
    p = q + std::strlen(s);
    return true;
  }
  void skip_ws() {
    while (p < t.size() && ws(t[p])) ++p;
  }
  bool name(std::string &out) {
    const size_t b = p;
    if (p >= t.size() || !name_start(static_cast<unsigned char>(t[p]))) return false;
    while (p < t.size() && name_char(static_cast<unsigned char>(t[p]))) ++p;
    out.assign(t, b, p - b);
    return true;
  }

  // After '<' of a start tag.
  bool element(XmlElem &e) {
    if (++depth > kMaxDepth) return fail("elements nested too deeply");
    const bool ok = element_body(e);
    --depth;
    return ok;
  }

  bool element_body(XmlElem &e) {
    if (!name(e.name)) return fail("bad element name");
    for (;;) {
      skip_ws();
      if (p >= t.size()) return fail("unterminated start tag");
      if (t[p] == '/') {
        if (p + 1 < t.size() && t[p + 1] == '>') {
          p += 2;
          return true;
        }
        return fail("bad empty-element tag");
      }
      if (t[p] == '>') {
        ++p;
        break;
      }
      XmlAttr a;
      if (!name(a.name)) return fail("bad attribute name");
      skip_ws();
      if (p >= t.size() || t[p] != '=') return fail("attribute without '='");
      ++p;
      skip_ws();
      if (p >= t.size() || (t[p] != '"' && t[p] != '\'')) return fail("attribute value not quoted");
      const char q = t[p++];
      const size_t end = t.find(q, p);
      if (end == std::string::npos) return fail("unterminated attribute value");
      a.value = decode(t.data() + p, end - p);
      p = end + 1;
      e.attrs.push_back(std::move(a));
    }
    // content
    for (;;) {
      const size_t lt = t.find('<', p);
      if (lt == std::string::npos) return fail("unclosed element");
      p = lt;
      if (starts("</")) {
        p += 2;
        std::string n;
        if (!name(n) || n != e.name) return fail("mismatched end tag");
        skip_ws();
        if (p >= t.size() || t[p] != '>') return fail("bad end tag");
        ++p;
        return true;
      }
      if (!misc()) {
        if (!err.empty()) return false;
        ++p;
        XmlElem c;
        if (!element(c)) return false;
        e.children.push_back(std::move(c));
      }
    }
  }

  // Comments, processing instructions, CDATA and DOCTYPE at p ('<'); true when one was skipped.
  bool misc() {
    if (starts("<?")) {
      if (!skip_past("?>")) return fail("unterminated declaration");
      return true;
    }
    if (starts("<!--")) {
      if (!skip_past("-->")) return fail("unterminated comment");
      return true;
    }
    if (starts("<![CDATA[")) {
      if (!skip_past("]]>")) return fail("unterminated CDATA");
      return true;
    }
    if (starts("<!")) {
      if (!skip_past(">")) return fail("unterminated declaration");
      return true;
    }
    return false;
  }
};

}  // namespace

bool parse_xml(const std::string &text, std::vector<XmlElem> &roots, std::string &err) {
  err.clear();
  Reader r(text, err);
  if (text.size() >= 3 && static_cast<unsigned char>(text[0]) == 0xEF &&
      static_cast<unsigned char>(text[1]) == 0xBB && static_cast<unsigned char>(text[2]) == 0xBF)
    r.p = 3;
  for (;;) {
    const size_t lt = text.find('<', r.p);
    if (lt == std::string::npos) break;
    r.p = lt;
    if (r.starts("</")) return r.fail("end tag without a start tag");
    if (r.misc()) continue;
    if (!err.empty()) return false;
    ++r.p;
    XmlElem e;
    if (!r.element(e)) return false;
    roots.push_back(std::move(e));
  }
  if (roots.empty()) {
    err = "no element";
    return false;
  }
  return true;
}

}  // namespace ingest
}  // namespace nomad
