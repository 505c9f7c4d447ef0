#include "xml.h"

#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>

namespace csmc {

const XmlNode *XmlNode::child(const std::string &n) const {
    for (const auto &c : children)
        if (!c->is_text && c->name == n) return c.get();
    return nullptr;
}

std::vector<const XmlNode *> XmlNode::children_named(const std::string &n) const {
    std::vector<const XmlNode *> out;
    for (const auto &c : children)
        if (!c->is_text && c->name == n) out.push_back(c.get());
    return out;
}

std::string XmlNode::attr(const std::string &n) const {
    for (const auto &a : attrs)
        if (a.first == n) return a.second;
    return "";
}

bool XmlNode::has_attr(const std::string &n) const {
    for (const auto &a : attrs)
        if (a.first == n) return true;
    return false;
}

std::string XmlNode::child_value() const {
    for (const auto &c : children)
        if (c->is_text) return c->text;
    return "";
}

std::string XmlNode::child_text(const std::string &n) const {
    const XmlNode *c = child(n);
    return c ? c->child_value() : std::string();
}

namespace {

bool is_space(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\r'; }

void append_utf8(std::string &out, unsigned long cp) {
    if (cp < 0x80) {
        out.push_back(static_cast<char>(cp));
    } else if (cp < 0x800) {
        out.push_back(static_cast<char>(0xC0 | (cp >> 6)));
        out.push_back(static_cast<char>(0x80 | (cp & 0x3F)));
    } else if (cp < 0x10000) {
        out.push_back(static_cast<char>(0xE0 | (cp >> 12)));
        out.push_back(static_cast<char>(0x80 | ((cp >> 6) & 0x3F)));
        out.push_back(static_cast<char>(0x80 | (cp & 0x3F)));
    } else {
        out.push_back(static_cast<char>(0xF0 | (cp >> 18)));
        out.push_back(static_cast<char>(0x80 | ((cp >> 12) & 0x3F)));
        out.push_back(static_cast<char>(0x80 | ((cp >> 6) & 0x3F)));
        out.push_back(static_cast<char>(0x80 | (cp & 0x3F)));
    }
}

class Parser {
  public:
    explicit Parser(const std::string &s) : s_(s) {}

    std::unique_ptr<XmlNode> document() {
        auto root = std::make_unique<XmlNode>();
        root->name = "#document";
        content(*root, /*top=*/true);
        return root;
    }

  private:
    const std::string &s_;
    size_t p_ = 0;

    [[noreturn]] void fail(const std::string &m) const {
        throw std::runtime_error("XML parse error at offset " + std::to_string(p_) + ": " + m);
    }
    bool starts(const char *t) const { return s_.compare(p_, std::strlen(t), t) == 0; }

    // Decodes entity references in [b, e) into out.
    void decode(size_t b, size_t e, std::string &out, bool attribute) const {
        for (size_t i = b; i < e; ++i) {
            char c = s_[i];
            if (c == '&') {
                size_t semi = s_.find(';', i);
                if (semi == std::string::npos || semi >= e) {
                    out.push_back('&');
                    continue;
                }
                std::string ent = s_.substr(i + 1, semi - i - 1);
                if (ent == "lt") out.push_back('<');
                else if (ent == "gt") out.push_back('>');
                else if (ent == "amp") out.push_back('&');
                else if (ent == "quot") out.push_back('"');
                else if (ent == "apos") out.push_back('\'');
                else if (!ent.empty() && ent[0] == '#') {
                    unsigned long cp = 0;
                    if (ent.size() > 1 && (ent[1] == 'x' || ent[1] == 'X'))
                        cp = std::strtoul(ent.c_str() + 2, nullptr, 16);
                    else
                        cp = std::strtoul(ent.c_str() + 1, nullptr, 10);
                    append_utf8(out, cp);
                } else {
                    out.append(s_, i, semi - i + 1);  // unknown entity kept verbatim
                }
                i = semi;
                continue;
            }
            if (c == '\r') {  // end-of-line normalisation
                if (i + 1 < e && s_[i + 1] == '\n') ++i;
                c = '\n';
            }
            if (attribute && (c == '\n' || c == '\t')) c = ' ';
            out.push_back(c);
        }
    }

    void skip_until(const char *term) {
        size_t q = s_.find(term, p_);
        if (q == std::string::npos) fail(std::string("unterminated construct, expected ") + term);
        p_ = q + std::strlen(term);
    }

    void skip_doctype() {  // <!DOCTYPE ... [ ... ]>
        int depth = 0;
        while (p_ < s_.size()) {
            char c = s_[p_++];
            if (c == '[') ++depth;
            else if (c == ']') --depth;
            else if (c == '>' && depth <= 0) return;
        }
        fail("unterminated DOCTYPE");
    }

    std::string name() {
        size_t b = p_;
        while (p_ < s_.size() && !is_space(s_[p_]) && s_[p_] != '>' && s_[p_] != '/' && s_[p_] != '=')
            ++p_;
        if (b == p_) fail("expected a name");
        return s_.substr(b, p_ - b);
    }

    void ws() {
        while (p_ < s_.size() && is_space(s_[p_])) ++p_;
    }

    void add_text(XmlNode &parent, size_t b, size_t e) {
        bool all_ws = true;
        for (size_t i = b; i < e; ++i)
            if (!is_space(s_[i])) { all_ws = false; break; }
        if (all_ws) return;
        auto t = std::make_unique<XmlNode>();
        t->is_text = true;
        decode(b, e, t->text, false);
        parent.children.push_back(std::move(t));
    }

    // Parses children of parent until its end tag (or end of input at top).
    void content(XmlNode &parent, bool top) {
        while (p_ < s_.size()) {
            size_t lt = s_.find('<', p_);
            if (lt == std::string::npos) {
                if (!top) fail("missing end tag for <" + parent.name + ">");
                add_text(parent, p_, s_.size());
                p_ = s_.size();
                return;
            }
            if (!top) add_text(parent, p_, lt);
            p_ = lt;
            if (starts("<!--")) { skip_until("-->"); continue; }
            if (starts("<![CDATA[")) {
                size_t b = p_ + 9;
                size_t q = s_.find("]]>", b);
                if (q == std::string::npos) fail("unterminated CDATA");
                auto t = std::make_unique<XmlNode>();
                t->is_text = true;
                for (size_t i = b; i < q; ++i) {
                    char c = s_[i];
                    if (c == '\r') { if (i + 1 < q && s_[i + 1] == '\n') ++i; c = '\n'; }
                    t->text.push_back(c);
                }
                if (!top) parent.children.push_back(std::move(t));
                p_ = q + 3;
                continue;
            }
            if (starts("<?")) { skip_until("?>"); continue; }
            if (starts("<!")) { skip_doctype(); continue; }
            if (starts("</")) {
                if (top) fail("unexpected end tag");
                p_ += 2;
                std::string n = name();
                if (n != parent.name) fail("end tag </" + n + "> does not match <" + parent.name + ">");
                ws();
                if (p_ >= s_.size() || s_[p_] != '>') fail("malformed end tag");
                ++p_;
                return;
            }
            // start tag
            ++p_;
            auto el = std::make_unique<XmlNode>();
            el->name = name();
            bool self_closing = false;
            for (;;) {
                ws();
                if (p_ >= s_.size()) fail("unterminated start tag");
                if (s_[p_] == '/') {
                    if (p_ + 1 < s_.size() && s_[p_ + 1] == '>') { p_ += 2; self_closing = true; break; }
                    fail("malformed start tag");
                }
                if (s_[p_] == '>') { ++p_; break; }
                std::string an = name();
                ws();
                if (p_ >= s_.size() || s_[p_] != '=') fail("expected '=' after attribute " + an);
                ++p_;
                ws();
                if (p_ >= s_.size() || (s_[p_] != '"' && s_[p_] != '\'')) fail("expected quoted value");
                char q = s_[p_++];
                size_t e = s_.find(q, p_);
                if (e == std::string::npos) fail("unterminated attribute value");
                std::string v;
                decode(p_, e, v, true);
                el->attrs.emplace_back(an, v);
                p_ = e + 1;
            }
            XmlNode *raw = el.get();
            parent.children.push_back(std::move(el));
            if (!self_closing) content(*raw, false);
        }
        if (!top) fail("missing end tag for <" + parent.name + ">");
    }
};

}  // namespace

std::unique_ptr<XmlNode> xml_parse(const std::string &text) {
    std::string s = text;
    // a UTF-8 byte-order mark before the declaration is not content
    if (s.size() >= 3 && (unsigned char)s[0] == 0xEF && (unsigned char)s[1] == 0xBB &&
        (unsigned char)s[2] == 0xBF)
        s.erase(0, 3);
    Parser p(s);
    return p.document();
}

std::unique_ptr<XmlNode> xml_parse_file(const std::string &path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("The specified file does not exist: " + path);
    std::stringstream ss;
    ss << f.rdbuf();
    return xml_parse(ss.str());
}

}  // namespace csmc
