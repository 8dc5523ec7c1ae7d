// Clean-room stand-in for the toml++ library (absent here), test infrastructure:
// the subset of its interface that SoL's scene loader uses
// (src/scene_loader.cpp, src/scene_loader.h), over a parser of our own for the
// TOML subset SoL's scene files use:
//
//   * comments (`#` to the end of the line, outside strings);
//   * `key = value` with bare or quoted keys;
//   * values: basic strings ("..." with \" \\ \n \t escapes), literal strings
//     ('...'), integers, floats (sign, fraction, exponent, inf, nan), booleans,
//     and arrays of these (nested arrays allowed, newlines inside arrays allowed);
//   * `[table]` and `[[array of tables]]` headers with single (undotted) names.
//
// Anything else is a parse error carrying the file and position, as toml++'s
// errors do.  Integers read through value_or<float> convert to float, which is
// what SoL's scene files rely on (e.g. `eye = [0, 0.9, 2.5]`).
#ifndef SOL_SHIM_TOML_H
#define SOL_SHIM_TOML_H

#include <cmath>
#include <cstdint>
#include <fstream>
#include <istream>
#include <iterator>
#include <memory>
#include <optional>
#include <sstream>
#include <stdexcept>
#include <string>
#include <string_view>
#include <type_traits>
#include <utility>
#include <variant>
#include <vector>

namespace toml {

struct source_position {
    size_t line = 0;
    size_t column = 0;
};

struct source_region {
    source_position begin;
    source_position end;
    std::shared_ptr<const std::string> path;
};

class parse_error : public std::runtime_error {
public:
    parse_error(const std::string& description, source_region region)
        : std::runtime_error(description), description_(description), region_(std::move(region)) {}
    std::string_view description() const noexcept { return description_; }
    const source_region& source() const noexcept { return region_; }

private:
    std::string description_;
    source_region region_;
};

class node;
class array;
class table;

template <typename Node>
class node_view;

/// An array of nodes.
class array {
public:
    std::vector<node> items;
    source_region region;

    size_t size() const { return items.size(); }
    auto begin() const { return items.begin(); }
    auto end() const { return items.end(); }
    node_view<const node> operator[](size_t i) const;
    const source_region& source() const { return region; }
};

/// A table: keys in insertion order.
class table {
public:
    std::vector<std::pair<std::string, node>> items;
    source_region region;

    node* find(std::string_view key);
    const node* find(std::string_view key) const;
    node_view<const node> operator[](std::string_view key) const;
    const source_region& source() const { return region; }
};

/// One value of the document.
class node {
public:
    using value_type = std::variant<std::monostate, std::string, int64_t, double, bool, std::shared_ptr<array>,
                                    std::shared_ptr<table>>;
    value_type v;
    source_region region;

    const table* as_table() const {
        auto p = std::get_if<std::shared_ptr<table>>(&v);
        return p ? p->get() : nullptr;
    }
    const array* as_array() const {
        auto p = std::get_if<std::shared_ptr<array>>(&v);
        return p ? p->get() : nullptr;
    }
    table* as_table() {
        auto p = std::get_if<std::shared_ptr<table>>(&v);
        return p ? p->get() : nullptr;
    }
    array* as_array() {
        auto p = std::get_if<std::shared_ptr<array>>(&v);
        return p ? p->get() : nullptr;
    }
    const source_region& source() const { return region; }

    /// The value as T if the node holds a T (integers also read as floats).
    template <typename T>
    std::optional<T> value() const {
        if constexpr (std::is_same_v<T, std::string> || std::is_same_v<T, std::string_view>) {
            if (auto s = std::get_if<std::string>(&v)) return T(*s);
        } else if constexpr (std::is_same_v<T, bool>) {
            if (auto b = std::get_if<bool>(&v)) return *b;
        } else if constexpr (std::is_floating_point_v<T>) {
            if (auto d = std::get_if<double>(&v)) return static_cast<T>(*d);
            if (auto i = std::get_if<int64_t>(&v)) return static_cast<T>(*i);
        } else if constexpr (std::is_integral_v<T>) {
            if (auto i = std::get_if<int64_t>(&v)) return static_cast<T>(*i);
        }
        return std::nullopt;
    }

    template <typename T>
    auto value_or(T&& fallback) const {
        using U = std::conditional_t<std::is_convertible_v<T, std::string_view> && !std::is_arithmetic_v<std::decay_t<T>>,
                                     std::string, std::decay_t<T>>;
        if (auto x = value<U>()) return *x;
        return U(std::forward<T>(fallback));
    }
};

/// A possibly empty reference to a node, as returned by table[key] and array[i].
template <typename Node>
class node_view {
public:
    node_view() = default;
    explicit node_view(Node* n) : n_(n) {}

    explicit operator bool() const { return n_ != nullptr; }
    Node* node() const { return n_; }

    const table* as_table() const { return n_ ? n_->as_table() : nullptr; }
    const array* as_array() const { return n_ ? n_->as_array() : nullptr; }

    template <typename T>
    std::optional<T> value() const {
        return n_ ? n_->template value<T>() : std::nullopt;
    }

    template <typename T>
    auto value_or(T&& fallback) const {
        using U = std::conditional_t<std::is_convertible_v<T, std::string_view> && !std::is_arithmetic_v<std::decay_t<T>>,
                                     std::string, std::decay_t<T>>;
        if (n_)
            if (auto x = n_->template value<U>()) return *x;
        return U(std::forward<T>(fallback));
    }

    node_view operator[](std::string_view key) const {
        const table* t = as_table();
        return node_view(t ? t->find(key) : nullptr);
    }
    node_view operator[](size_t i) const {
        const array* a = as_array();
        return node_view(a && i < a->items.size() ? &a->items[i] : nullptr);
    }

private:
    Node* n_ = nullptr;
};

inline node_view<const node> array::operator[](size_t i) const {
    return node_view<const node>(i < items.size() ? &items[i] : nullptr);
}

inline node* table::find(std::string_view key) {
    for (auto& kv : items)
        if (kv.first == key) return &kv.second;
    return nullptr;
}

inline const node* table::find(std::string_view key) const {
    for (auto& kv : items)
        if (kv.first == key) return &kv.second;
    return nullptr;
}

inline node_view<const node> table::operator[](std::string_view key) const {
    return node_view<const node>(find(key));
}

namespace detail {

/// Recursive-descent reader over the whole document.
class reader {
public:
    reader(std::string text, std::shared_ptr<const std::string> path) : s_(std::move(text)), path_(std::move(path)) {}

    table parse() {
        table root;
        root.region = region();
        table* current = &root;
        while (true) {
            skip_ws_comments_newlines();
            if (eof()) break;
            if (peek() == '[') {
                const bool array_of_tables = peek(1) == '[';
                const source_region at = region();
                pos_ += array_of_tables ? 2 : 1;
                col_ += array_of_tables ? 2 : 1;
                skip_ws();
                std::string name = key();
                skip_ws();
                expect(']');
                if (array_of_tables) expect(']');
                end_of_line();
                if (array_of_tables) {
                    node* n = root.find(name);
                    if (!n) {
                        root.items.emplace_back(name, node{});
                        n = &root.items.back().second;
                        n->v = std::make_shared<array>();
                        n->region = at;
                        n->as_array()->region = at;
                    }
                    array* a = n->as_array();
                    if (!a) fail("'" + name + "' is not an array of tables", at);
                    a->items.emplace_back();
                    node& t = a->items.back();
                    t.v = std::make_shared<table>();
                    t.region = at;
                    t.as_table()->region = at;
                    current = t.as_table();
                } else {
                    if (root.find(name)) fail("redefinition of table '" + name + "'", at);
                    root.items.emplace_back(name, node{});
                    node& t = root.items.back().second;
                    t.v = std::make_shared<table>();
                    t.region = at;
                    t.as_table()->region = at;
                    current = t.as_table();
                }
                continue;
            }
            const source_region at = region();
            std::string k = key();
            skip_ws();
            expect('=');
            skip_ws();
            node value = parse_value();
            value.region = at;
            if (current->find(k)) fail("redefinition of key '" + k + "'", at);
            current->items.emplace_back(std::move(k), std::move(value));
            end_of_line();
        }
        return root;
    }

private:
    std::string s_;
    std::shared_ptr<const std::string> path_;
    size_t pos_ = 0, line_ = 1, col_ = 1;

    bool eof() const { return pos_ >= s_.size(); }
    char peek(size_t k = 0) const { return pos_ + k < s_.size() ? s_[pos_ + k] : '\0'; }
    char get() {
        const char c = s_[pos_++];
        if (c == '\n') { ++line_; col_ = 1; } else { ++col_; }
        return c;
    }
    source_region region() const {
        source_region r;
        r.begin = {line_, col_};
        r.end = r.begin;
        r.path = path_;
        return r;
    }
    [[noreturn]] void fail(const std::string& what) const { throw parse_error(what, region()); }
    [[noreturn]] void fail(const std::string& what, const source_region& at) const { throw parse_error(what, at); }
    void expect(char c) {
        if (peek() != c) fail(std::string("expected '") + c + "'");
        get();
    }
    void skip_ws() {
        while (!eof() && (peek() == ' ' || peek() == '\t')) get();
    }
    void skip_comment() {
        if (peek() == '#')
            while (!eof() && peek() != '\n') get();
    }
    void skip_ws_comments_newlines() {
        while (!eof()) {
            const char c = peek();
            if (c == ' ' || c == '\t' || c == '\r' || c == '\n') get();
            else if (c == '#') skip_comment();
            else break;
        }
    }
    void end_of_line() {
        skip_ws();
        skip_comment();
        if (peek() == '\r') get();
        if (!eof() && peek() != '\n') fail("unexpected text after a value");
    }
    static bool bare_key_char(char c) {
        return (c >= 'a' && c <= 'z') || (c >= 'A' && c <= 'Z') || (c >= '0' && c <= '9') || c == '_' || c == '-';
    }
    std::string key() {
        if (peek() == '"') return basic_string();
        if (peek() == '\'') return literal_string();
        std::string k;
        while (!eof() && bare_key_char(peek())) k += get();
        if (k.empty()) fail("expected a key");
        return k;
    }
    std::string basic_string() {
        expect('"');
        std::string out;
        while (true) {
            if (eof() || peek() == '\n') fail("unterminated string");
            char c = get();
            if (c == '"') break;
            if (c == '\\') {
                const char e = eof() ? '\0' : get();
                switch (e) {
                    case '"': out += '"'; break;
                    case '\\': out += '\\'; break;
                    case 'n': out += '\n'; break;
                    case 't': out += '\t'; break;
                    case 'r': out += '\r'; break;
                    default: fail("unsupported escape sequence");
                }
            } else {
                out += c;
            }
        }
        return out;
    }
    std::string literal_string() {
        expect('\'');
        std::string out;
        while (true) {
            if (eof() || peek() == '\n') fail("unterminated string");
            char c = get();
            if (c == '\'') break;
            out += c;
        }
        return out;
    }
    node number() {
        std::string text;
        while (!eof()) {
            const char c = peek();
            if ((c >= '0' && c <= '9') || c == '+' || c == '-' || c == '.' || c == 'e' || c == 'E' || c == '_' ||
                c == 'i' || c == 'n' || c == 'f' || c == 'a')
                text += get();
            else
                break;
        }
        std::string clean;
        for (char c : text)
            if (c != '_') clean += c;
        node n;
        if (clean == "inf" || clean == "+inf") { n.v = HUGE_VAL; return n; }
        if (clean == "-inf") { n.v = -HUGE_VAL; return n; }
        if (clean == "nan" || clean == "+nan" || clean == "-nan") { n.v = std::nan(""); return n; }
        const bool is_float = clean.find_first_of(".eE") != std::string::npos;
        size_t used = 0;
        try {
            if (is_float) n.v = std::stod(clean, &used);
            else n.v = static_cast<int64_t>(std::stoll(clean, &used, 10));
        } catch (const std::exception&) {
            fail("invalid number '" + text + "'");
        }
        if (used != clean.size() || clean.empty()) fail("invalid number '" + text + "'");
        return n;
    }
    node parse_value() {
        const char c = peek();
        node n;
        if (c == '"') { n.v = basic_string(); return n; }
        if (c == '\'') { n.v = literal_string(); return n; }
        if (c == '[') {
            const source_region at = region();
            get();
            auto a = std::make_shared<array>();
            a->region = at;
            while (true) {
                skip_ws_comments_newlines();
                if (peek() == ']') { get(); break; }
                node item = parse_value();
                item.region = at;
                a->items.push_back(std::move(item));
                skip_ws_comments_newlines();
                if (peek() == ',') { get(); continue; }
                if (peek() == ']') { get(); break; }
                fail("expected ',' or ']' in an array");
            }
            n.v = a;
            return n;
        }
        if (s_.compare(pos_, 4, "true") == 0) { for (int i = 0; i < 4; ++i) get(); n.v = true; return n; }
        if (s_.compare(pos_, 5, "false") == 0) { for (int i = 0; i < 5; ++i) get(); n.v = false; return n; }
        if ((c >= '0' && c <= '9') || c == '+' || c == '-' || c == 'i' || c == 'n') return number();
        fail("unsupported value");
    }
};

}  // namespace detail

/// Parses a document; throws parse_error on malformed input.
inline table parse(std::istream& is, std::string_view source_path = {}) {
    std::string text((std::istreambuf_iterator<char>(is)), std::istreambuf_iterator<char>());
    detail::reader r(std::move(text), std::make_shared<const std::string>(source_path));
    return r.parse();
}

inline table parse(std::string_view doc, std::string_view source_path = {}) {
    detail::reader r(std::string(doc), std::make_shared<const std::string>(source_path));
    return r.parse();
}

}  // namespace toml

#endif
