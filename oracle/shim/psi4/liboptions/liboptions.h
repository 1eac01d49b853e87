/*
 * Oracle shim (test infrastructure only): a Psi4-style Options object holding
 * the option values that the reference hot-path sources query.
 */
#ifndef ORACLE_SHIM_LIBOPTIONS_H
#define ORACLE_SHIM_LIBOPTIONS_H

#include <map>
#include <string>
#include <vector>

namespace psi {

class Data {
  public:
    Data() = default;
    explicit Data(double v) : value_(v) {}
    bool has_changed() const { return changed_; }
    int size() const { return (int)array_.size(); }
    double to_double() const { return value_; }
    Data& operator[](int i) { return array_[i]; }

    bool changed_ = false;
    double value_ = 0.0;
    std::vector<Data> array_;
};

class Options {
  public:
    bool get_bool(const std::string& k) const { return num_.at(k) != 0.0; }
    int get_int(const std::string& k) const { return (int)num_.at(k); }
    double get_double(const std::string& k) const { return num_.at(k); }
    std::string get_str(const std::string& k) const { return str_.at(k); }
    Data& operator[](const std::string& k) { return data_[k]; }

    void set_num(const std::string& k, double v) { num_[k] = v; }
    void set_str(const std::string& k, const std::string& v) { str_[k] = v; }

  private:
    std::map<std::string, double> num_;
    std::map<std::string, std::string> str_;
    std::map<std::string, Data> data_;
};

}  // namespace psi

#endif
