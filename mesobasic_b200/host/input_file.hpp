// Reader of mesoBasic's input-parameter file (input.dat) with the lookup
// semantics of the GetPot calls the reference makes (GetPot file in
// src/utils; used by MesoExecute.cpp:59-101, PFApp.cpp:17-29 and the model
// constructors):
//   - the file is split into whitespace-separated tokens; '#' starts a
//     comment that runs to the end of the line; 'single quotes' group a
//     token that holds spaces;
//   - a token "=" joins its neighbours into one "name=value" argument;
//   - [Name] opens section "Name/", [] returns to the top level, [./Sub]
//     opens "Sub/" inside the current section and [../] leaves one level;
//   - a variable defined twice takes the later value;
//   - sections are listed in order of first appearance;
//   - numbers are read as sscanf("%lf") would; an int is that double
//     truncated, so "2.0e1" reads as 20; an unreadable number gives the
//     caller's default.
// Command-line arguments of the form name=value (e.g. Domain/nx=128) are
// applied after the file, so they override it.
#pragma once

#include <string>
#include <utility>
#include <vector>

class InputFile {
public:
    InputFile() = default;
    // throws std::runtime_error when the file cannot be read
    explicit InputFile(const std::string& path);
    static InputFile from_text(const std::string& text);

    // name=value overrides (later ones win)
    void set(const std::string& name, const std::string& value);

    int operator()(const char* name, int def) const;
    double operator()(const char* name, double def) const;
    std::string operator()(const char* name, const char* def) const;
    bool has(const char* name) const;

    // section prefixes ("Domain/", "PFApp/", ...) in order of appearance
    const std::vector<std::string>& section_names() const { return sections_; }
    const std::vector<std::pair<std::string, std::string>>& variables() const { return vars_; }

private:
    void parse(const std::string& text);
    const std::string* find(const std::string& name) const;

    std::vector<std::pair<std::string, std::string>> vars_;
    std::vector<std::string> sections_;
};
