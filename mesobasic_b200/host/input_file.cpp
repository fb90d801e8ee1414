// See input_file.hpp.
#include "input_file.hpp"

#include <algorithm>
#include <cstdio>
#include <fstream>
#include <sstream>
#include <stdexcept>

namespace {

// whitespace-separated tokens, '#' comments, 'quoted' tokens
std::vector<std::string> tokenize(const std::string& text)
{
    std::vector<std::string> out;
    size_t i = 0, n = text.size();
    while (i < n) {
        const char ch = text[i];
        if (ch == '#') {
            while (i < n && text[i] != '\n') ++i;
            continue;
        }
        if (ch == ' ' || ch == '\t' || ch == '\n' || ch == '\r' || ch == '\f' || ch == '\v') {
            ++i;
            continue;
        }
        std::string tok;
        while (i < n) {
            const char c = text[i];
            if (c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\f' || c == '\v' || c == '#') break;
            if (c == '\'') {  // quoted run, quotes dropped
                ++i;
                while (i < n && text[i] != '\'') tok += text[i++];
                if (i < n) ++i;
                continue;
            }
            tok += c;
            ++i;
        }
        out.push_back(tok);
    }
    return out;
}

// join  a = b  /  a= b  /  a =b  into one "a=b" argument
std::vector<std::string> join_assignments(const std::vector<std::string>& t)
{
    std::vector<std::string> out;
    for (size_t i = 0; i < t.size(); ++i) {
        std::string a = t[i];
        if (i + 1 < t.size() && t[i + 1] == "=") {
            a += "=";
            if (i + 2 < t.size()) a += t[i + 2];
            i += 2;
        } else if (!a.empty() && a.back() == '=' && a.size() > 1 && a[0] != '[' && i + 1 < t.size()) {
            a += t[++i];
        } else if (i + 1 < t.size() && t[i + 1].size() > 1 && t[i + 1][0] == '=' && a.find('=') == std::string::npos &&
                   a[0] != '[') {
            a += t[++i];
        }
        out.push_back(a);
    }
    return out;
}

}  // namespace

InputFile::InputFile(const std::string& path)
{
    std::ifstream f(path);
    if (!f) throw std::runtime_error("cannot read input file '" + path + "'");
    std::stringstream ss;
    ss << f.rdbuf();
    parse(ss.str());
}

InputFile InputFile::from_text(const std::string& text)
{
    InputFile in;
    in.parse(text);
    return in;
}

void InputFile::parse(const std::string& text)
{
    std::vector<std::string> stack;  // section path components
    std::string section;
    for (const std::string& arg : join_assignments(tokenize(text))) {
        if (arg.size() > 1 && arg.front() == '[' && arg.back() == ']') {
            std::string label = arg.substr(1, arg.size() - 2);
            if (label.empty()) {
                stack.clear();
            } else if (label.rfind("./", 0) == 0 || label.rfind("../", 0) == 0) {
                // relative label: ./ stays, each ../ pops one level
                while (!label.empty()) {
                    if (label.rfind("./", 0) == 0) {
                        label.erase(0, 2);
                    } else if (label.rfind("../", 0) == 0) {
                        label.erase(0, 3);
                        if (!stack.empty()) stack.pop_back();
                    } else {
                        break;
                    }
                }
                if (!label.empty()) {
                    if (label.back() == '/') label.pop_back();
                    stack.push_back(label);
                }
            } else {
                if (label.back() == '/') label.pop_back();
                stack.assign(1, label);
            }
            section.clear();
            for (const std::string& s : stack) section += s + "/";
            if (!section.empty() && std::find(sections_.begin(), sections_.end(), section) == sections_.end())
                sections_.push_back(section);
            continue;
        }
        const size_t eq = arg.find('=');
        if (eq == std::string::npos || eq == 0) continue;  // bare words carry no variable
        set(section + arg.substr(0, eq), arg.substr(eq + 1));
    }
}

void InputFile::set(const std::string& name, const std::string& value)
{
    for (auto& kv : vars_)
        if (kv.first == name) {
            kv.second = value;
            return;
        }
    vars_.emplace_back(name, value);
}

const std::string* InputFile::find(const std::string& name) const
{
    for (const auto& kv : vars_)
        if (kv.first == name) return &kv.second;
    return nullptr;
}

bool InputFile::has(const char* name) const { return find(name) != nullptr; }

double InputFile::operator()(const char* name, double def) const
{
    const std::string* v = find(name);
    if (!v) return def;
    double d;
    if (std::sscanf(v->c_str(), "%lf", &d) != 1) return def;
    return d;
}

int InputFile::operator()(const char* name, int def) const
{
    return (int)(*this)(name, (double)def);
}

std::string InputFile::operator()(const char* name, const char* def) const
{
    const std::string* v = find(name);
    return v ? *v : std::string(def);
}
