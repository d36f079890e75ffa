// Command-line options with the reference's parser semantics
// (lib/cmdline as extended by src/util/cmdline_hooks.cpp), shared by the
// drop-in commands.
#pragma once

#include <cmath>
#include <cstdlib>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

namespace strip_cli {

// ---------------------------------------------------------------------------
// options: the reference's option set (options.cpp:13-76, reconstruction_cmd
// .cpp:114-115, common/options.cpp:5-20) and its parser semantics
// (lib/cmdline: --name=value, --name value, -x value, -abc flags; config
// files hold one argument per line, '#' lines ignored; options marked
// not_from_file ignore config files).
// ---------------------------------------------------------------------------
struct Option {
  std::string name;
  char short_name;
  bool has_value;
  bool not_from_file;
  std::string def;
  std::string help;
  std::string value;
  int count = 0;
};

class Options {
 public:
  // the scanner, common and OpenMP options of both commands
  // (options.cpp:13-43, common/options.cpp:5-20)
  void add_scanner_options() {
    add("config", 'c', true, false, "", "load config file");
    add("radius", 'r', true, false, "0.5", "R distance between scintillator");
    add("length", 'l', true, false, "1", "scintillator length");
    add("s-pixel", 'p', true, false, "0.01", "pixel size");
    add("n-pixels", 'n', true, false, "0", "number of pixels");
    add("n-z-pixels", 0, true, false, "", "number of z pixels");
    add("n-y-pixels", 0, true, false, "", "number of y pixels");
    add("s-z", 0, true, false, "0.015", "TOF sigma along z axis");
    add("s-dl", 0, true, false, "0.06", "TOF sigma delta-l");
    add("n-emissions", 'e', true, true, "0", "number of emissions");
    add("verbose", 'v', false, false, "", "print progress information (-v) or benchmark (-vv)");
    add("n-threads", 'T', true, false, "", "number of host threads");
    add("help", 'h', false, false, "", "print this message");
  }

  // Command-line errors throw; in config files they are collected into
  // *errors (cmdline_hooks.cpp:84-92 reports them as warnings).
  void parse(const std::vector<std::string>& args, bool from_file,
             std::vector<std::string>* errors = nullptr) {
    for (size_t i = 0; i < args.size(); ++i) {
      try {
        parse_one(args, i, from_file);
      } catch (const std::string& e) {
        if (!errors) throw;
        errors->push_back(e);
      }
    }
  }

  void parse_one(const std::vector<std::string>& args, size_t& i, bool from_file) {
    {
      const std::string& a = args[i];
      if (a.compare(0, 2, "--") == 0) {
        const auto eq = a.find('=');
        const std::string name = a.substr(2, eq == std::string::npos ? std::string::npos : eq - 2);
        Option& o = get(name);
        if (eq != std::string::npos) {
          set(o, a.substr(eq + 1), from_file);
        } else if (o.has_value) {
          if (i + 1 >= args.size()) throw std::string("option needs value: --") + name;
          set(o, args[++i], from_file);
        } else {
          set(o, "", from_file);
        }
      } else if (a.size() > 1 && a[0] == '-') {
        for (size_t j = 1; j < a.size(); ++j) {
          Option& o = get_short(a[j]);
          const bool last = j + 1 == a.size();
          if (last && o.has_value && i + 1 < args.size()) {
            set(o, args[++i], from_file);
          } else if (o.has_value) {
            throw std::string("option needs value: -") + a[j];
          } else {
            set(o, "", from_file);
          }
        }
      } else if (a != "-") {
        rest.push_back(a);
      }
    }
  }

  // cmdline::load (cmdline_hooks.cpp:50-96): relative paths resolve against
  // the including config file's directory.
  void load(const std::string& arg) {
    std::string path = arg;
    if (!dir_stack_.empty() && !path.empty() && path[0] != '/')
      path = dir_stack_.back() + path;
    if (exist("verbose")) std::cout << "# load: " << path << std::endl;
    std::ifstream in(path);
    if (!in.is_open()) throw "cannot open input config file: " + path;
    const auto sep = path.find_last_of('/');
    dir_stack_.push_back(sep == std::string::npos ? std::string() : path.substr(0, sep + 1));
    std::vector<std::string> lines;
    std::string line;
    while (std::getline(in, line))
      if (!line.empty() && line[0] != '#') lines.push_back(line);
    const size_t n_rest = rest.size();
    std::vector<std::string> errors;
    parse(lines, true, &errors);
    rest.resize(n_rest);  // positional lines of a config file are ignored
    if (!errors.empty()) {
      std::cerr << (errors.size() == 1 ? "warning" : "warnings") << " parsing " << path
                << ":" << std::endl;
      for (const auto& e : errors) std::cerr << "  " << e << std::endl;
    }
    dir_stack_.pop_back();
  }

  bool exist(const std::string& name) const { return opts_.at(name).count > 0; }
  int count(const std::string& name) const { return opts_.at(name).count; }
  std::string str(const std::string& name) const {
    const Option& o = opts_.at(name);
    return o.count ? o.value : o.def;
  }
  double num(const std::string& name) const {
    const std::string s = str(name);
    // vector options (--radius) keep their first comma-separated element
    return std::strtod(s.substr(0, s.find(',')).c_str(), nullptr);
  }
  int integer(const std::string& name) const { return (int)std::strtol(str(name).c_str(), nullptr, 10); }
  void set_int(const std::string& name, int v) {
    Option& o = opts_.at(name);
    o.value = std::to_string(v);
    if (!o.count) o.count = 1;
  }

  std::string usage(const char* prog, const char* rest_name = "response") const {
    std::ostringstream os;
    os << "usage: " << prog << " [options] ... " << rest_name << " ...\n"
       << "note: All length options below should be expressed in milimeters.\n"
       << "options:\n";
    for (const auto& name : order_) {
      const Option& o = opts_.at(name);
      os << "  ";
      if (o.short_name) os << "-" << o.short_name << ", "; else os << "    ";
      os << "--" << std::left << std::setw(16) << o.name << o.help;
      if (o.has_value && !o.def.empty()) os << " (=" << o.def << ")";
      os << "\n";
    }
    return os.str();
  }

  std::vector<std::string> rest;

  void add(const std::string& name, char s, bool has_value, bool nff,
           const std::string& def, const std::string& help) {
    Option o;
    o.name = name;
    o.short_name = s;
    o.has_value = has_value;
    o.not_from_file = nff;
    o.def = def;
    o.help = help;
    opts_[name] = o;
    order_.push_back(name);
  }

  // "--name=value" / "--name" lines of the options that were given, as
  // cmdline's operator<< saves a configuration (lib/cmdline/cmdline.h:717,
  // 868-960; options listed in `always` are saved with their defaults too)
  void save(std::ostream& os, const std::vector<std::string>& skip,
            const std::vector<std::string>& always) const {
    for (const auto& name : order_) {
      const Option& o = opts_.at(name);
      bool skipped = false, forced = false;
      for (const auto& k : skip) skipped |= k == name;
      for (const auto& k : always) forced |= k == name;
      if (skipped || (!o.count && !forced)) continue;
      if (o.has_value) os << "--" << name << "=" << (o.count ? o.value : o.def) << "\n";
      else os << "--" << name << "\n";
    }
  }

 private:
  Option& get(const std::string& name) {
    auto it = opts_.find(name);
    if (it == opts_.end()) throw "undefined option: --" + name;
    return it->second;
  }
  Option& get_short(char c) {
    for (auto& kv : opts_)
      if (kv.second.short_name == c) return kv.second;
    throw std::string("undefined short option: -") + c;
  }
  void set(Option& o, const std::string& v, bool from_file) {
    if (from_file && o.not_from_file) return;
    if (o.name == "config") {
      load(v);
      return;
    }
    o.value = v;
    ++o.count;
  }

  std::map<std::string, Option> opts_;
  std::vector<std::string> order_;
  std::vector<std::string> dir_stack_;
};


// calculate_scanner_options (options.cpp:106-124): -n sets both pixel
// counts, otherwise missing counts follow from length / pixel and 2R / pixel.
inline void calculate_scanner_options(Options& cl) {
  if (cl.exist("n-pixels")) {
    cl.set_int("n-z-pixels", cl.integer("n-pixels"));
    cl.set_int("n-y-pixels", cl.integer("n-pixels"));
  } else {
    if (!cl.exist("n-z-pixels"))
      cl.set_int("n-z-pixels", (int)std::ceil(cl.num("length") / cl.num("s-pixel")));
    if (!cl.exist("n-y-pixels"))
      cl.set_int("n-y-pixels", (int)std::ceil(2 * cl.num("radius") / cl.num("s-pixel")));
  }
}

// counts accept k, m, g suffixes (util/cmdline_types.h:114-137)
inline long long parse_count(const std::string& s) {
  char* end = nullptr;
  long long v = std::strtoll(s.c_str(), &end, 10);
  if (end && end[0] && !end[1]) {
    switch (end[0]) {
      case 'k': case 'K': v *= 1000; break;
      case 'm': case 'M': v *= 1000000; break;
      case 'g': case 'G': v *= 1000000000; break;
      default: throw "invalid count: " + s;
    }
  } else if (end && end[0]) {
    throw "invalid count: " + s;
  }
  return v;
}

}  // namespace strip_cli
