// vah_properties.h -- reader for the reference's .properties files.
//
// The reference reads rhic-conf/{lattice,ic,hydro}.properties with libconfig
// 1.5 (Properties.cpp:10-22 over config_lookup_int / config_lookup_float).
// libconfig is not a dependency here; this reader accepts the subset of its
// grammar those files use -- `name = value` or `name: value`, optional `;` or
// `,` terminator, `#`, `//` and `/* */` comments, integer (decimal, hex, L
// suffix), float, boolean and string scalars -- and keeps libconfig's typing:
// without auto-conversion an integer literal does not answer a float lookup,
// nor a float literal an integer lookup.
#pragma once

#include <map>
#include <string>

namespace vah {

struct Setting {
    enum Type { INT, FLOAT, BOOL, STRING } type;
    long long i = 0;
    double f = 0.0;
    bool b = false;
    std::string s;
};

class Properties {
  public:
    // Parse a file; false (with a message in *err) if it is missing or malformed.
    bool read_file(const std::string &path, std::string *err);
    bool read_string(const std::string &text, std::string *err);

    bool lookup_int(const std::string &name, int *out) const;
    bool lookup_float(const std::string &name, double *out) const;
    bool lookup_bool(const std::string &name, bool *out) const;
    bool lookup_string(const std::string &name, std::string *out) const;
    bool auto_convert = false;  // libconfig's CONFIG_OPTION_AUTOCONVERT (off by default)

    const std::map<std::string, Setting> &settings() const { return map_; }

  private:
    std::map<std::string, Setting> map_;
};

}  // namespace vah
