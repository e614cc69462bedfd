// Drop-in for DENSE's `csv_gen` (source/csv_gen.cpp): writes the three
// parameter-file templates of the model this binary is linked with,
// param_sets_template.csv, param_pert_template.csv and
// param_grad_template.csv, into the directory given as the first argument
// (a prefix, as DENSE uses it: "dir/" + file name).  The column headers come
// from the engine library's model tables (dense_model_*_name); the text of
// the files is DENSE's, since users and DENSE's readers rely on it.
// DENSE writes "rcrit_" twice before a critical species' name (csv_gen.cpp
// prefixes a list whose entries already carry it); kept, so the files match.

#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "dense_b200.h"

namespace {

const char* const kGreen = "\x1b[32m";
const char* const kRed = "\x1b[31m";
const char* const kReset = "\x1b[0m";

enum class Kind { kSets, kPert, kGrad };

void write_template(const std::string& path, Kind kind, const dense_model_info& info) {
  std::ofstream out(path);
  if (!out.is_open()) {
    std::cout << kRed << "CSV file output failed. CSV file '" << path << "' unable to be written to." << kReset
              << '\n';
  }
  out << "# CSV Specification\n"
         "#   Ignored by the file readers are:\n"
         "#     (1) Empty cells / Blank rows / Whitespace\n"
         "#     (2) Comment whose rows always begin with a '#'\n"
         "#         For best results delete all comments before loading this file into any Excel-like program.\n"
         "#     (3) Any cell which does not conform to the scientific notation format 3.14e-41 or simple whole "
         "numbers and decimals\n"
         "#         Often times cells which do not contain numbers are intended to be column headers. These are "
         "not parsed by the simulation and can technically be modified by the users as they wish.\n"
         "#         It is futile to add/remove/modify the column headers with the expectation of changing the "
         "program's behavior. Data must be entered in the default order for it to be parsed correctly.\n"
         "# None of these comments include commas because it messes with the column widths when loaded into "
         "Excel-like programs.\n"
         "# For more information and examples see README.md section 2.2.0\n";
  out << "\n# Rename this file by removing the \"_template\" from the file name (or just change the name "
         "entirely) once the data has been entered!\n";
  std::vector<std::string> prefix;
  std::string what;
  switch (kind) {
    case Kind::kSets:
      out << "# This file can contain more than one set (each being on their own line). All sets are "
             "initialized and executed in parallel when a file is loaded into the simulation.\n";
      out << "# For more information and examples see README.md section 2.2.1\n\n";
      what = "sets";
      prefix = {""};
      break;
    case Kind::kPert:
      out << "# This file should only contain one set of perturbations. Only this one perturbations set is "
             "applied to all parameter sets when a simulation set is being run.\n";
      out << "# Use '0' to indicate that a reaction should not have perturbations.\n";
      out << "# For more information and examples see README.md section 2.2.2\n\n";
      what = "perturbations";
      prefix = {"pert_"};
      break;
    case Kind::kGrad:
      out << "# This file should only contain one set of gradients. Only this one gradients setting is "
             "applied to all parameter sets when a simulation set is being run.\n";
      out << "# Use '0' under all four columns of a reaction to indiate that it should not have a gradient.\n"
             "# Gradient Codes\n"
             "#   x1 - start column\n"
             "#   y1 - start multiplier (use '1.23' to mean '123%')\n"
             "#   x2 - end column\n"
             "#   y2 - end multiplier\n";
      out << "# For more information and examples see README.md section 2.2.2\n\n";
      what = "gradients";
      prefix = {"grad_x1_", "grad_y1_", "grad_x2_", "grad_y2_"};
      break;
  }
  std::string zeros = "\n";
  auto columns = [&](const std::string& name) {
    for (const auto& p : prefix) {
      out << p << name << ", ";
      zeros += "0, ";
    }
    if (kind == Kind::kGrad) {  // a blank column between a parameter's four
      out << ", ";
      zeros += ", ";
    }
  };
  for (int r = 0; r < info.num_reactions; ++r) columns(dense_model_reaction_name(r));
  out << ", ";
  zeros += ", ";
  for (int d = 0; d < info.num_delay_reactions; ++d)
    columns(std::string("dreact_") + dense_model_delay_reaction_name(d));
  out << ", ";
  zeros += ", ";
  for (int c = 0; c < info.num_critical_species; ++c)
    columns(std::string("rcrit_rcrit_") + dense_model_critical_specie_name(c));
  if (kind != Kind::kSets) out << zeros;
  std::cout << kGreen << "CSV parameter " << what << " column header generation successful. See '" << path
            << "'.\n"
            << kReset;
}

}  // namespace

int main(int argc, char* argv[]) {
  if (argc < 2) {
    std::cout << kRed
              << "CSV parameter list column header generation failed. Missing required command line argument:\n"
                 "\t(1) Relative directory containing desired model files, such as \"../models/her_model_2014/\", "
                 "not including quotation marks. Spaces not allowed in file/directory names. For indicating the "
                 "current directory, use \"./\".\n"
              << kReset;
    return EXIT_FAILURE;
  }
  dense_model_info info{};
  if (dense_model_get_info(&info) != DENSE_OK) {
    std::cout << kRed << "model tables unavailable: " << dense_last_error() << kReset << '\n';
    return EXIT_FAILURE;
  }
  const std::string dir = argv[1];
  write_template(dir + "param_sets_template.csv", Kind::kSets, info);
  write_template(dir + "param_pert_template.csv", Kind::kPert, info);
  write_template(dir + "param_grad_template.csv", Kind::kGrad, info);
  return EXIT_SUCCESS;
}
