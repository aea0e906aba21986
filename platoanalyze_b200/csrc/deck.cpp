// Input decks: XML reader and Teuchos-style parameter tree (see deck.hpp).
#include "deck.hpp"

#include <cctype>
#include <cerrno>
#include <cstdlib>
#include <fstream>
#include <sstream>

namespace plato::deck {

namespace {

std::string trim(const std::string& s) {
    size_t b = 0, e = s.size();
    while (b < e && std::isspace(static_cast<unsigned char>(s[b]))) ++b;
    while (e > b && std::isspace(static_cast<unsigned char>(s[e - 1]))) --e;
    return s.substr(b, e - b);
}

void append_utf8(std::string& out, unsigned long cp) {
    if (cp < 0x80) {
        out += char(cp);
    } else if (cp < 0x800) {
        out += char(0xC0 | (cp >> 6));
        out += char(0x80 | (cp & 0x3F));
    } else if (cp < 0x10000) {
        out += char(0xE0 | (cp >> 12));
        out += char(0x80 | ((cp >> 6) & 0x3F));
        out += char(0x80 | (cp & 0x3F));
    } else {
        out += char(0xF0 | (cp >> 18));
        out += char(0x80 | ((cp >> 12) & 0x3F));
        out += char(0x80 | ((cp >> 6) & 0x3F));
        out += char(0x80 | (cp & 0x3F));
    }
}

std::string decode_entities(const std::string& s) {
    std::string out;
    out.reserve(s.size());
    for (size_t i = 0; i < s.size(); ++i) {
        if (s[i] != '&') {
            out += s[i];
            continue;
        }
        const size_t semi = s.find(';', i);
        if (semi == std::string::npos) throw DeckError("XML: unterminated entity reference");
        const std::string ent = s.substr(i + 1, semi - i - 1);
        if (ent == "lt") out += '<';
        else if (ent == "gt") out += '>';
        else if (ent == "amp") out += '&';
        else if (ent == "quot") out += '"';
        else if (ent == "apos") out += '\'';
        else if (!ent.empty() && ent[0] == '#') {
            const bool hex = ent.size() > 1 && (ent[1] == 'x' || ent[1] == 'X');
            const std::string digits = ent.substr(hex ? 2 : 1);
            char* end = nullptr;
            const unsigned long cp = std::strtoul(digits.c_str(), &end, hex ? 16 : 10);
            if (digits.empty() || *end != '\0') throw DeckError("XML: bad character reference &" + ent + ";");
            append_utf8(out, cp);
        } else {
            throw DeckError("XML: unknown entity &" + ent + ";");
        }
        i = semi;
    }
    return out;
}

class XmlReader {
public:
    explicit XmlReader(const std::string& t) : s_(t) {}

    XmlNode document() {
        XmlNode wrapper;
        for (;;) {
            skip_misc();
            if (p_ >= s_.size()) break;
            if (s_[p_] != '<') throw error("text outside the root element");
            wrapper.children.push_back(element());
        }
        if (wrapper.children.empty()) throw DeckError("XML: no element");
        if (wrapper.children.size() == 1) return std::move(wrapper.children[0]);
        return wrapper;
    }

private:
    DeckError error(const std::string& what) const {
        size_t line = 1;
        for (size_t i = 0; i < p_ && i < s_.size(); ++i) line += s_[i] == '\n';
        return DeckError("XML line " + std::to_string(line) + ": " + what);
    }
    bool starts(const char* lit) const { return s_.compare(p_, std::char_traits<char>::length(lit), lit) == 0; }
    void skip_ws() {
        while (p_ < s_.size() && std::isspace(static_cast<unsigned char>(s_[p_]))) ++p_;
    }
    void skip_past(const char* end) {
        const size_t q = s_.find(end, p_);
        if (q == std::string::npos) throw error(std::string("missing '") + end + "'");
        p_ = q + std::char_traits<char>::length(end);
    }
    // whitespace, comments, processing instructions, DOCTYPE
    void skip_misc() {
        for (;;) {
            skip_ws();
            if (starts("<!--")) skip_past("-->");
            else if (starts("<?")) skip_past("?>");
            else if (starts("<!DOCTYPE")) skip_past(">");
            else return;
        }
    }
    std::string name() {
        const size_t b = p_;
        while (p_ < s_.size() && (std::isalnum(static_cast<unsigned char>(s_[p_])) || s_[p_] == '_' || s_[p_] == '-' ||
                                  s_[p_] == ':' || s_[p_] == '.'))
            ++p_;
        if (p_ == b) throw error("expected a name");
        return s_.substr(b, p_ - b);
    }
    XmlNode element() {
        ++p_;  // '<'
        XmlNode n;
        n.tag = name();
        for (;;) {
            skip_ws();
            if (p_ >= s_.size()) throw error("unterminated start tag <" + n.tag + ">");
            if (starts("/>")) {
                p_ += 2;
                return n;
            }
            if (s_[p_] == '>') {
                ++p_;
                break;
            }
            std::string key = name();
            skip_ws();
            if (p_ >= s_.size() || s_[p_] != '=') throw error("expected '=' after attribute " + key);
            ++p_;
            skip_ws();
            if (p_ >= s_.size() || (s_[p_] != '\'' && s_[p_] != '"')) throw error("attribute value must be quoted");
            const char q = s_[p_++];
            const size_t e = s_.find(q, p_);
            if (e == std::string::npos) throw error("unterminated attribute value");
            for (const auto& a : n.attrs)
                if (a.first == key) throw error("duplicate attribute " + key);
            n.attrs.emplace_back(key, decode_entities(s_.substr(p_, e - p_)));
            p_ = e + 1;
        }
        std::string text;
        for (;;) {
            if (p_ >= s_.size()) throw error("unterminated element <" + n.tag + ">");
            if (starts("<!--")) {
                skip_past("-->");
            } else if (starts("<![CDATA[")) {
                p_ += 9;
                const size_t e = s_.find("]]>", p_);
                if (e == std::string::npos) throw error("unterminated CDATA");
                text += s_.substr(p_, e - p_);
                p_ = e + 3;
            } else if (starts("<?")) {
                skip_past("?>");
            } else if (starts("</")) {
                p_ += 2;
                const std::string closing = name();
                if (closing != n.tag) throw error("</" + closing + "> closes <" + n.tag + ">");
                skip_ws();
                if (p_ >= s_.size() || s_[p_] != '>') throw error("malformed end tag");
                ++p_;
                n.text = trim(text);
                return n;
            } else if (s_[p_] == '<') {
                n.children.push_back(element());
            } else {
                const size_t e = s_.find('<', p_);
                if (e == std::string::npos) throw error("unterminated element <" + n.tag + ">");
                text += decode_entities(s_.substr(p_, e - p_));
                p_ = e;
            }
        }
    }

    const std::string& s_;
    size_t p_ = 0;
};

std::vector<std::string> split_array(const std::string& raw, const std::string& key) {
    std::string v = trim(raw);
    if (v.size() < 2 || v.front() != '{' || v.back() != '}')
        throw DeckError("parameter '" + key + "': array value must be written {a, b, ...}");
    v = v.substr(1, v.size() - 2);
    std::vector<std::string> out;
    if (trim(v).empty()) return out;
    std::stringstream ss(v);
    std::string item;
    while (std::getline(ss, item, ',')) out.push_back(trim(item));
    return out;
}

double to_double(const std::string& raw, const std::string& key) {
    const std::string v = trim(raw);
    char* end = nullptr;
    errno = 0;
    const double d = std::strtod(v.c_str(), &end);
    if (v.empty() || *end != '\0' || errno == ERANGE) throw DeckError("parameter '" + key + "': not a number: " + v);
    return d;
}

int to_int(const std::string& raw, const std::string& key) {
    const std::string v = trim(raw);
    char* end = nullptr;
    errno = 0;
    const long d = std::strtol(v.c_str(), &end, 10);
    if (v.empty() || *end != '\0' || errno == ERANGE || d < -2147483648L || d > 2147483647L)
        throw DeckError("parameter '" + key + "': not an integer: " + v);
    return int(d);
}

void fill_list(ParamList& L, const XmlNode& node) {
    for (const XmlNode& c : node.children) {
        const std::string* nm = c.attr("name");
        if (c.tag == "ParameterList") {
            if (!nm) throw DeckError("ParameterList without a name inside '" + L.name + "'");
            if (L.has(*nm)) throw DeckError("'" + *nm + "' defined twice in '" + L.name + "'");
            ParamEntry e;
            e.list = std::make_shared<ParamList>();
            e.list->name = *nm;
            fill_list(*e.list, c);
            L.entries.emplace_back(*nm, std::move(e));
        } else if (c.tag == "Parameter") {
            const std::string* ty = c.attr("type");
            const std::string* va = c.attr("value");
            if (!nm || !ty || !va) throw DeckError("Parameter needs name, type and value in '" + L.name + "'");
            if (L.has(*nm)) throw DeckError("'" + *nm + "' defined twice in '" + L.name + "'");
            ParamEntry e;
            e.type = *ty;
            e.value = *va;
            L.entries.emplace_back(*nm, std::move(e));
        }
        // other elements (e.g. Validators) carry no parameters
    }
}

const XmlNode* find_param_list(const XmlNode& n) {
    if (n.tag == "ParameterList") return &n;
    for (const XmlNode& c : n.children)
        if (const XmlNode* f = find_param_list(c)) return f;
    return nullptr;
}

}  // namespace

const std::string* XmlNode::attr(const std::string& name) const {
    for (const auto& a : attrs)
        if (a.first == name) return &a.second;
    return nullptr;
}

std::vector<const XmlNode*> XmlNode::children_named(const std::string& t) const {
    std::vector<const XmlNode*> out;
    for (const XmlNode& c : children)
        if (c.tag == t) out.push_back(&c);
    return out;
}

std::string XmlNode::child_text(const std::string& t, const std::string& fallback) const {
    for (const XmlNode& c : children)
        if (c.tag == t) return c.text;
    return fallback;
}

bool XmlNode::has_child(const std::string& t) const {
    for (const XmlNode& c : children)
        if (c.tag == t) return true;
    return false;
}

XmlNode parse_xml(const std::string& text) { return XmlReader(text).document(); }

const ParamEntry* ParamList::find(const std::string& key) const {
    for (const auto& e : entries)
        if (e.first == key) return &e.second;
    return nullptr;
}

bool ParamList::is_sublist(const std::string& key) const {
    const ParamEntry* e = find(key);
    return e && e->is_list();
}

const ParamList& ParamList::sublist(const std::string& key) const {
    const ParamEntry* e = find(key);
    if (!e || !e->is_list()) throw DeckError("sublist '" + key + "' missing in '" + name + "'");
    return *e->list;
}

static const ParamEntry& scalar_entry(const ParamList& L, const std::string& key) {
    const ParamEntry* e = L.find(key);
    if (!e) throw DeckError("parameter '" + key + "' missing in '" + L.name + "'");
    if (e->is_list()) throw DeckError("'" + key + "' in '" + L.name + "' is a sublist, not a parameter");
    return *e;
}

std::string ParamList::get_string(const std::string& key) const { return scalar_entry(*this, key).value; }
std::string ParamList::get_string(const std::string& key, const std::string& fallback) const {
    return has(key) ? get_string(key) : fallback;
}
double ParamList::get_double(const std::string& key) const { return to_double(scalar_entry(*this, key).value, key); }
double ParamList::get_double(const std::string& key, double fallback) const {
    return has(key) ? get_double(key) : fallback;
}
int ParamList::get_int(const std::string& key) const { return to_int(scalar_entry(*this, key).value, key); }
int ParamList::get_int(const std::string& key, int fallback) const { return has(key) ? get_int(key) : fallback; }

bool ParamList::get_bool(const std::string& key, bool fallback) const {
    if (!has(key)) return fallback;
    std::string v = trim(scalar_entry(*this, key).value);
    for (char& c : v) c = char(std::tolower(static_cast<unsigned char>(c)));
    if (v == "true" || v == "1" || v == "yes") return true;
    if (v == "false" || v == "0" || v == "no") return false;
    throw DeckError("parameter '" + key + "': not a bool: " + v);
}

std::vector<double> ParamList::get_double_array(const std::string& key) const {
    std::vector<double> out;
    for (const std::string& item : split_array(scalar_entry(*this, key).value, key)) out.push_back(to_double(item, key));
    return out;
}

std::vector<std::string> ParamList::get_string_array(const std::string& key) const {
    return split_array(scalar_entry(*this, key).value, key);
}

bool ParamList::is_type(const std::string& key, const std::string& type) const {
    const ParamEntry* e = find(key);
    return e && !e->is_list() && e->type == type;
}

void ParamList::set_target(const std::string& target, double value) {
    std::vector<std::string> tokens;
    std::stringstream ss(target);
    std::string item;
    while (std::getline(ss, item, ':')) tokens.push_back(item);
    if (tokens.empty()) throw DeckError("empty parameter target");
    ParamList* L = this;
    size_t i = 0;
    for (; i + 1 < tokens.size() && tokens[i].size() >= 2 && tokens[i].front() == '[' && tokens[i].back() == ']'; ++i) {
        const std::string name = tokens[i].substr(1, tokens[i].size() - 2);
        ParamEntry* found = nullptr;
        for (auto& e : L->entries)
            if (e.first == name) found = &e.second;
        if (!found || !found->is_list()) throw DeckError("target '" + target + "': no sublist '" + name + "'");
        L = found->list.get();
    }
    if (i + 1 != tokens.size()) throw DeckError("target '" + target + "': sublists must be written [name]");
    std::ostringstream v;
    v.precision(17);
    v << value;
    const std::string& last = tokens.back();
    const size_t p1 = last.find('('), p2 = last.find(')');
    if (p1 != std::string::npos && p2 != std::string::npos && p2 > p1) {
        const std::string name = last.substr(0, p1);
        const int idx = to_int(last.substr(p1 + 1, p2 - p1 - 1), target);
        for (auto& e : L->entries) {
            if (e.first != name) continue;
            if (e.second.is_list()) break;
            std::vector<std::string> items = split_array(e.second.value, name);
            if (idx < 0 || size_t(idx) >= items.size()) throw DeckError("target '" + target + "': index out of range");
            items[size_t(idx)] = v.str();
            std::string joined = "{";
            for (size_t k = 0; k < items.size(); ++k) joined += (k ? ", " : "") + items[k];
            e.second.value = joined + "}";
            return;
        }
        throw DeckError("target '" + target + "': no array '" + name + "'");
    }
    for (auto& e : L->entries)
        if (e.first == last) {
            if (e.second.is_list()) throw DeckError("target '" + target + "' is a sublist");
            e.second.type = "double";
            e.second.value = v.str();
            return;
        }
    ParamEntry e;
    e.type = "double";
    e.value = v.str();
    L->entries.emplace_back(last, std::move(e));
}

std::shared_ptr<ParamList> to_param_list(const XmlNode& root) {
    const XmlNode* pl = find_param_list(root);
    if (!pl) throw DeckError("no ParameterList element");
    auto L = std::make_shared<ParamList>();
    const std::string* nm = pl->attr("name");
    L->name = nm ? *nm : std::string();
    fill_list(*L, *pl);
    return L;
}

std::shared_ptr<ParamList> parse_param_list(const std::string& xml_text) { return to_param_list(parse_xml(xml_text)); }

std::string read_file(const std::string& path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw DeckError("cannot open '" + path + "'");
    std::stringstream ss;
    ss << f.rdbuf();
    return ss.str();
}

}  // namespace plato::deck
