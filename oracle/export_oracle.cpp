// TEST INFRASTRUCTURE ONLY — never linked into or called by the product path.
//
// C++ restatement of the reference connector's three output writers
// (src/connector/connector.cuh: export_results_csv :839-904,
// export_time_series_csv :906-932, export_structured_json :934-1155) written
// through real std::ofstream objects, so the stream's carried-over float format
// and uppercase flag behave exactly as in the reference. It checks the
// Python exporter bk_b200.export, which emulates that stream state.
//
// Usage: export_oracle <records.txt> <results.csv> <time_series.csv> <structured.json> [n_override]
// Records file: whitespace-separated tokens; per record "R" then the fields in
// the order read by read_record(); strings as "<len> <token>" ('-' when empty),
// vectors as "<count> v...", maps as "<count> k v ...".
#include <cstdint>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <sstream>
#include <string>
#include <utility>
#include <vector>

namespace {

struct Rec {
  int n = 0;
  double g = 0.0;
  size_t trap_rank = 0;
  uint64_t trap_bits = 0;
  int64_t trap_energy = 0;
  int d_min = 0;
  std::string canonical_id, canonical_hex, canonical_bitstring;
  double window_avg_p_less = 0, window_avg_dh = 0, initial_rise_rate_avg = 0, initial_rise_rate_max = 0;
  double quantum_time_sec = 0;
  std::vector<double> time_points, p_less_history, dh_history;
  double p_blind = 0, peak_p_less = 0, peak_time = 0;
  int num_sampling_seeds = 1;
  std::vector<uint64_t> sample_seeds;
  std::vector<double> sample_success_rates;
  std::vector<size_t> sample_improved_shots, sample_total_shots;
  std::vector<int64_t> sample_best_energies;
  std::vector<double> sample_mean_hamming_flips;
  int best_d = 0;
  double best_d_rate = 0;
  size_t best_d_successes = 0, best_d_trials = 0, best_d_evals = 0;
  std::map<int, double> rate_by_d;
  std::map<int, size_t> trials_by_d, evals_by_d;
  double kick_time_sec = 0;
  double restart_rate = 0;
  size_t restart_successes = 0, restart_trials = 0, restart_evals = 0;
  double restart_time_sec = 0;
  double tabu_direct_rate = 0;
  size_t tabu_direct_successes = 0, tabu_direct_trials = 0, tabu_direct_evals = 0;
  double tabu_direct_time_sec = 0;
  int tabu_kick_d = 0;
  double tabu_kick_rate = 0;
  size_t tabu_kick_successes = 0, tabu_kick_trials = 0, tabu_kick_evals = 0;
  std::map<int, double> tabu_rate_by_d;
  std::map<int, size_t> tabu_trials_by_d, tabu_evals_by_d;
  double tabu_kick_time_sec = 0;
  double tabu_restart_rate = 0;
  size_t tabu_restart_successes = 0, tabu_restart_trials = 0, tabu_restart_evals = 0;
  double tabu_restart_time_sec = 0;
  double tabu_best_rate = 0;
  std::string tabu_best_method;
  size_t sd_total_evaluations = 0, tabu_total_evaluations = 0, total_evaluations = 0;
};

std::string rd_str(std::istream& in) {
  size_t len;
  std::string tok;
  in >> len >> tok;
  return len == 0 ? std::string() : tok;
}
template <class T>
std::vector<T> rd_vec(std::istream& in) {
  size_t c;
  in >> c;
  std::vector<T> v(c);
  for (auto& x : v) in >> x;
  return v;
}
template <class V>
std::map<int, V> rd_map(std::istream& in) {
  size_t c;
  in >> c;
  std::map<int, V> m;
  for (size_t i = 0; i < c; ++i) {
    int k;
    V v;
    in >> k >> v;
    m[k] = v;
  }
  return m;
}

bool read_record(std::istream& in, Rec& r) {
  std::string tag;
  if (!(in >> tag)) return false;
  if (tag != "R") return false;
  in >> r.n >> r.g >> r.trap_rank >> r.trap_bits >> r.trap_energy >> r.d_min;
  r.canonical_id = rd_str(in);
  r.canonical_hex = rd_str(in);
  r.canonical_bitstring = rd_str(in);
  in >> r.window_avg_p_less >> r.window_avg_dh >> r.initial_rise_rate_avg >> r.initial_rise_rate_max >>
      r.quantum_time_sec;
  r.time_points = rd_vec<double>(in);
  r.p_less_history = rd_vec<double>(in);
  r.dh_history = rd_vec<double>(in);
  in >> r.p_blind >> r.peak_p_less >> r.peak_time >> r.num_sampling_seeds;
  r.sample_seeds = rd_vec<uint64_t>(in);
  r.sample_success_rates = rd_vec<double>(in);
  r.sample_improved_shots = rd_vec<size_t>(in);
  r.sample_total_shots = rd_vec<size_t>(in);
  r.sample_best_energies = rd_vec<int64_t>(in);
  r.sample_mean_hamming_flips = rd_vec<double>(in);
  in >> r.best_d >> r.best_d_rate >> r.best_d_successes >> r.best_d_trials >> r.best_d_evals;
  r.rate_by_d = rd_map<double>(in);
  r.trials_by_d = rd_map<size_t>(in);
  r.evals_by_d = rd_map<size_t>(in);
  in >> r.kick_time_sec >> r.restart_rate >> r.restart_successes >> r.restart_trials >> r.restart_evals >>
      r.restart_time_sec;
  in >> r.tabu_direct_rate >> r.tabu_direct_successes >> r.tabu_direct_trials >> r.tabu_direct_evals >>
      r.tabu_direct_time_sec;
  in >> r.tabu_kick_d >> r.tabu_kick_rate >> r.tabu_kick_successes >> r.tabu_kick_trials >> r.tabu_kick_evals;
  r.tabu_rate_by_d = rd_map<double>(in);
  r.tabu_trials_by_d = rd_map<size_t>(in);
  r.tabu_evals_by_d = rd_map<size_t>(in);
  in >> r.tabu_kick_time_sec >> r.tabu_restart_rate >> r.tabu_restart_successes >> r.tabu_restart_trials >>
      r.tabu_restart_evals >> r.tabu_restart_time_sec >> r.tabu_best_rate;
  r.tabu_best_method = rd_str(in);
  in >> r.sd_total_evaluations >> r.tabu_total_evaluations >> r.total_evaluations;
  return static_cast<bool>(in);
}

// connector.cuh:906-932
void time_series(std::ostream& f, const std::vector<Rec>& rs) {
  f << "N,g,trap_rank,trap_energy,time,p_less,dH,p_blind\n";
  for (const auto& r : rs) {
    for (size_t i = 0; i < r.time_points.size() && i < r.p_less_history.size(); ++i) {
      const double dh = i < r.dh_history.size() ? r.dh_history[i] : 0.0;
      f << r.n << "," << r.g << "," << r.trap_rank << "," << r.trap_energy << "," << std::fixed
        << std::setprecision(4) << r.time_points[i] << "," << std::scientific << std::setprecision(6)
        << r.p_less_history[i] << "," << std::fixed << std::setprecision(4) << dh << "," << std::scientific
        << std::setprecision(6) << r.p_blind << "\n";
    }
  }
}

// connector.cuh:839-904
void results(std::ostream& f, const std::vector<Rec>& rs) {
  f << "N,g,trap_rank,canonical_id,canonical_hex,trap_energy,d_min,window_avg_p_less,window_avg_dh,"
    << "initial_rise_rate_avg,initial_rise_rate_max,peak_p_less,peak_time,p_blind,"
    << "best_d,best_d_rate,best_d_successes,best_d_trials,best_d_evals,"
    << "restart_rate,restart_successes,restart_trials,restart_evals,"
    << "tabu_best_method,tabu_best_rate,tabu_direct_rate,tabu_kick_d,tabu_kick_rate,tabu_restart_rate,"
    << "sd_total_evaluations,tabu_total_evaluations,total_evaluations,"
    << "quantum_time_sec,kick_time_sec,restart_time_sec,tabu_kick_time_sec,"
    << "sample_seed1_rate,sample_seed2_rate,sample_seed3_rate,trap_bits\n";
  for (const auto& r : rs) {
    auto rate = [&](size_t k) { return r.sample_success_rates.size() > k ? r.sample_success_rates[k] : 0.0; };
    f << r.n << "," << r.g << "," << r.trap_rank << "," << r.canonical_id << "," << r.canonical_hex << ","
      << r.trap_energy << "," << r.d_min << "," << std::scientific << std::setprecision(6) << r.window_avg_p_less
      << "," << std::fixed << std::setprecision(4) << r.window_avg_dh << "," << std::scientific
      << std::setprecision(6) << r.initial_rise_rate_avg << "," << std::scientific << std::setprecision(6)
      << r.initial_rise_rate_max << "," << r.peak_p_less << "," << std::fixed << std::setprecision(4)
      << r.peak_time << "," << std::scientific << std::setprecision(6) << r.p_blind << "," << r.best_d << ","
      << r.best_d_rate << "," << r.best_d_successes << "," << r.best_d_trials << "," << r.best_d_evals << ","
      << r.restart_rate << "," << r.restart_successes << "," << r.restart_trials << "," << r.restart_evals << ","
      << "\"" << r.tabu_best_method << "\"," << r.tabu_best_rate << "," << r.tabu_direct_rate << ","
      << r.tabu_kick_d << "," << r.tabu_kick_rate << "," << r.tabu_restart_rate << "," << r.sd_total_evaluations
      << "," << r.tabu_total_evaluations << "," << r.total_evaluations << "," << std::fixed << std::setprecision(4)
      << r.quantum_time_sec << "," << r.kick_time_sec << "," << r.restart_time_sec << "," << r.tabu_kick_time_sec
      << "," << std::scientific << std::setprecision(6) << rate(0) << "," << std::scientific << std::setprecision(6)
      << rate(1) << "," << std::scientific << std::setprecision(6) << rate(2) << ","
      << "0x" << std::hex << std::uppercase << r.trap_bits << std::dec << "\n";
  }
}

template <class M>
void map_f(std::ostream& f, const char* name, const M& m) {
  f << "        \"" << name << "\": {";
  size_t di = 0;
  for (const auto& kv : m) {
    f << (di > 0 ? ", " : "") << "\"" << kv.first << "\": " << std::scientific << std::setprecision(6) << kv.second;
    ++di;
  }
  f << "},\n";
}
template <class M>
void map_i(std::ostream& f, const char* name, const M& m) {
  f << "        \"" << name << "\": {";
  size_t di = 0;
  for (const auto& kv : m) {
    f << (di > 0 ? ", " : "") << "\"" << kv.first << "\": " << kv.second;
    ++di;
  }
  f << "},\n";
}
template <class V, class F>
void arr(std::ostream& f, const V& v, F&& put) {
  for (size_t i = 0; i < v.size(); ++i) {
    f << (i > 0 ? ", " : "");
    put(v[i]);
  }
}

// connector.cuh:934-1155
void structured(std::ostream& f, const std::vector<Rec>& rs, int n_override) {
  std::map<std::pair<int, size_t>, std::vector<Rec>> groups;
  for (const auto& r : rs) groups[{r.n, r.trap_rank}].push_back(r);
  int sys_n = n_override;
  if (sys_n == 0 && !rs.empty()) sys_n = rs.front().n;
  f << "{\n  \"system\": {\n    \"N\": " << sys_n << ",\n    \"num_seeds\": " << groups.size() << "\n  },\n";
  f << "  \"seeds\": [\n";
  size_t ti = 0;
  for (auto it = groups.begin(); it != groups.end(); ++it, ++ti) {
    const auto& lst = it->second;
    const Rec& a = lst.front();
    f << "    {\n";
    f << "      \"N\": " << a.n << ",\n";
    f << "      \"trap_rank\": " << a.trap_rank << ",\n";
    f << "      \"canonical_id\": \"" << a.canonical_id << "\",\n";
    f << "      \"canonical_hex\": \"" << a.canonical_hex << "\",\n";
    f << "      \"canonical_bitstring\": \"" << a.canonical_bitstring << "\",\n";
    f << "      \"trap_state_hex\": \"0x" << std::hex << std::uppercase << a.trap_bits << std::dec << "\",\n";
    f << "      \"trap_energy_E0\": " << a.trap_energy << ",\n";
    f << "      \"d_min\": " << a.d_min << ",\n";
    f << "      \"classical_baselines\": {\n";
    f << "        \"best_d\": " << a.best_d << ",\n";
    f << "        \"best_d_rate\": " << std::scientific << std::setprecision(6) << a.best_d_rate << ",\n";
    f << "        \"best_d_successes\": " << a.best_d_successes << ",\n";
    f << "        \"best_d_trials\": " << a.best_d_trials << ",\n";
    f << "        \"best_d_evals\": " << a.best_d_evals << ",\n";
    map_f(f, "rates_by_d", a.rate_by_d);
    map_i(f, "trials_by_d", a.trials_by_d);
    map_i(f, "evals_by_d", a.evals_by_d);
    f << "        \"restart_rate\": " << std::scientific << std::setprecision(6) << a.restart_rate << ",\n";
    f << "        \"restart_successes\": " << a.restart_successes << ",\n";
    f << "        \"restart_trials\": " << a.restart_trials << ",\n";
    f << "        \"restart_evals\": " << a.restart_evals << ",\n";
    f << "        \"sd_total_evaluations\": " << a.sd_total_evaluations << ",\n";
    f << "        \"tabu_direct_rate\": " << std::scientific << std::setprecision(6) << a.tabu_direct_rate << ",\n";
    f << "        \"tabu_direct_successes\": " << a.tabu_direct_successes << ",\n";
    f << "        \"tabu_direct_trials\": " << a.tabu_direct_trials << ",\n";
    f << "        \"tabu_direct_evals\": " << a.tabu_direct_evals << ",\n";
    f << "        \"tabu_kick_d\": " << a.tabu_kick_d << ",\n";
    f << "        \"tabu_kick_rate\": " << std::scientific << std::setprecision(6) << a.tabu_kick_rate << ",\n";
    f << "        \"tabu_kick_successes\": " << a.tabu_kick_successes << ",\n";
    f << "        \"tabu_kick_trials\": " << a.tabu_kick_trials << ",\n";
    f << "        \"tabu_kick_evals\": " << a.tabu_kick_evals << ",\n";
    map_f(f, "tabu_rates_by_d", a.tabu_rate_by_d);
    map_i(f, "tabu_trials_by_d", a.tabu_trials_by_d);
    map_i(f, "tabu_evals_by_d", a.tabu_evals_by_d);
    f << "        \"tabu_restart_rate\": " << std::scientific << std::setprecision(6) << a.tabu_restart_rate << ",\n";
    f << "        \"tabu_restart_successes\": " << a.tabu_restart_successes << ",\n";
    f << "        \"tabu_restart_trials\": " << a.tabu_restart_trials << ",\n";
    f << "        \"tabu_restart_evals\": " << a.tabu_restart_evals << ",\n";
    f << "        \"tabu_best_rate\": " << std::scientific << std::setprecision(6) << a.tabu_best_rate << ",\n";
    f << "        \"tabu_best_method\": \"" << a.tabu_best_method << "\",\n";
    f << "        \"tabu_total_evaluations\": " << a.tabu_total_evaluations << ",\n";
    f << "        \"total_evaluations\": " << a.total_evaluations << ",\n";
    f << "        \"kick_time_sec\": " << std::fixed << std::setprecision(4) << a.kick_time_sec << ",\n";
    f << "        \"restart_time_sec\": " << std::fixed << std::setprecision(4) << a.restart_time_sec << ",\n";
    f << "        \"tabu_direct_time_sec\": " << std::fixed << std::setprecision(4) << a.tabu_direct_time_sec
      << ",\n";
    f << "        \"tabu_kick_time_sec\": " << std::fixed << std::setprecision(4) << a.tabu_kick_time_sec << ",\n";
    f << "        \"tabu_restart_time_sec\": " << std::fixed << std::setprecision(4) << a.tabu_restart_time_sec
      << "\n";
    f << "      },\n";
    f << "      \"quantum_dynamics\": {\n";
    for (size_t gi = 0; gi < lst.size(); ++gi) {
      const Rec& q = lst[gi];
      std::ostringstream gs;
      gs << std::fixed << std::setprecision(2) << q.g;
      f << "        \"" << gs.str() << "\": {\n";
      f << "          \"g\": " << std::fixed << std::setprecision(2) << q.g << ",\n";
      f << "          \"window_avg_p_less\": " << std::scientific << std::setprecision(6) << q.window_avg_p_less
        << ",\n";
      f << "          \"window_avg_dH\": " << std::fixed << std::setprecision(4) << q.window_avg_dh << ",\n";
      f << "          \"initial_rise_rate_avg\": " << std::scientific << std::setprecision(6)
        << q.initial_rise_rate_avg << ",\n";
      f << "          \"initial_rise_rate_max\": " << std::scientific << std::setprecision(6)
        << q.initial_rise_rate_max << ",\n";
      f << "          \"peak_p_less\": " << std::scientific << std::setprecision(6) << q.peak_p_less << ",\n";
      f << "          \"peak_time\": " << std::fixed << std::setprecision(4) << q.peak_time << ",\n";
      f << "          \"p_blind\": " << std::scientific << std::setprecision(6) << q.p_blind << ",\n";
      f << "          \"time_array\": [";
      arr(f, q.time_points, [&](double x) { f << std::fixed << std::setprecision(4) << x; });
      f << "],\n          \"p_less_array\": [";
      arr(f, q.p_less_history, [&](double x) { f << std::scientific << std::setprecision(6) << x; });
      f << "],\n          \"dH_array\": [";
      arr(f, q.dh_history, [&](double x) { f << std::fixed << std::setprecision(4) << x; });
      f << "],\n";
      f << "          \"quantum_time_sec\": " << std::fixed << std::setprecision(4) << q.quantum_time_sec << ",\n";
      f << "          \"sampling_validation\": {\n";
      f << "            \"num_sampling_seeds\": " << q.num_sampling_seeds << ",\n";
      f << "            \"seeds\": [";
      arr(f, q.sample_seeds, [&](uint64_t x) { f << x; });
      f << "],\n            \"sample_success_rates\": [";
      arr(f, q.sample_success_rates, [&](double x) { f << std::scientific << std::setprecision(6) << x; });
      f << "],\n            \"sample_improved_shots\": [";
      arr(f, q.sample_improved_shots, [&](size_t x) { f << x; });
      f << "],\n            \"sample_total_shots\": [";
      arr(f, q.sample_total_shots, [&](size_t x) { f << x; });
      f << "],\n            \"sample_best_energies\": [";
      arr(f, q.sample_best_energies, [&](int64_t x) { f << x; });
      f << "],\n            \"sample_mean_hamming_flips\": [";
      arr(f, q.sample_mean_hamming_flips, [&](double x) { f << std::fixed << std::setprecision(4) << x; });
      f << "]\n          }\n";
      f << "        }" << (gi + 1 < lst.size() ? "," : "") << "\n";
    }
    f << "      }\n";
    f << "    }" << (ti + 1 < groups.size() ? "," : "") << "\n";
  }
  f << "  ]\n}\n";
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 5) {
    std::cerr << "usage: export_oracle records results.csv time_series.csv structured.json [n_override]\n";
    return 2;
  }
  std::ifstream in(argv[1]);
  std::vector<Rec> rs;
  Rec r;
  while (read_record(in, r)) {
    rs.push_back(r);
    r = Rec();
  }
  const int n_override = argc > 5 ? std::stoi(argv[5]) : 0;
  std::ofstream f1(argv[2]), f2(argv[3]), f3(argv[4]);
  results(f1, rs);
  time_series(f2, rs);
  structured(f3, rs, n_override);
  std::cout << rs.size() << " records\n";
  return 0;
}
