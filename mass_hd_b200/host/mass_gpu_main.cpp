// mass-gpu: standalone driver for the GPU model plugins.
//
// Runs a MASS runcard the way the reference's `mass` program does
// (src/main.cpp:132-345, src/options.cpp:38-216, src/write.cpp:28-195):
//   mass-gpu runcard.dat [-o dir] [--key=value ...] [--no-write] [-f]
// The runcard holds `key = value` lines (# starts a comment); command-line
// --key=value pairs take precedence over the runcard. The model is built by
// name through the plugin registry, then Initialize(), Configure(),
// parameters.json, and the time loop: frame<t>.json every ninfo steps from
// nstart on, Step() x nsubsteps, RuntimeChecks() every ninfo steps, and a
// final frame<nsteps>.json. Output files have the reference's names and
// JSON layout, so massPy's loadarchive reads them.
//
// The reference's `-t` (OpenMP threads) is accepted and ignored; zip
// compression is not provided. --save-state=<file> writes the device state
// at the end of the run as a full-precision checkpoint (mass_lb_save), which
// a lattice of the same model and size loads with mass_lb_load.
#include "header.hpp"
#include "models.hpp"
#include "error_msg.hpp"
#include "random.hpp"
#include "lyotropic_gpu.hpp"
#include "nematic_gpu.hpp"
#include "mass_lb_ext.h"

#include <chrono>
#include <fstream>
#include <thread>
#include <sys/stat.h>

using namespace std;

unsigned nsubsteps = 1;

namespace {

struct Program
{
  string runname = "./", model_name, inputname, save_state;
  unsigned LX = 0, LY = 0, nsteps = 0, ninfo = 1, nstart = 0, BC = 0, seed = 0;
  bool has_seed = false, no_write = false, no_warning = false, stop_at_warning = false;
  bool force_delete = false;
  unsigned verbose = 1;
};

string trim(const string& s)
{
  const auto a = s.find_first_not_of(" \t\r\n");
  if(a == string::npos) return "";
  const auto b = s.find_last_not_of(" \t\r\n");
  return s.substr(a, b - a + 1);
}

vector<pair<string, string>> read_runcard(const string& path)
{
  ifstream in(path);
  if(!in.good()) throw error_msg("can not open runcard file ", path);
  vector<pair<string, string>> kv;
  string line;
  while(getline(in, line))
  {
    const auto h = line.find('#');
    if(h != string::npos) line = line.substr(0, h);
    const auto eq = line.find('=');
    if(eq == string::npos) continue;
    const string k = trim(line.substr(0, eq)), v = trim(line.substr(eq + 1));
    if(!k.empty()) kv.emplace_back(k, v);
  }
  return kv;
}

template<class T>
void to(const string& text, T& out, const string& key)
{
  istringstream is(text);
  T v{};
  is >> v;
  if(is.fail()) throw error_msg("invalid value '", text, "' for option ", key);
  out = v;
}

bool set_program_option(Program& p, const string& k, const string& v)
{
  if(k == "output" || k == "o") p.runname = v;
  else if(k == "model" || k == "m") p.model_name = v;
  else if(k == "LX") to(v, p.LX, k);
  else if(k == "LY") to(v, p.LY, k);
  else if(k == "nsteps") to(v, p.nsteps, k);
  else if(k == "nsubsteps") to(v, nsubsteps, k);
  else if(k == "ninfo") to(v, p.ninfo, k);
  else if(k == "seed") { to(v, p.seed, k); p.has_seed = true; }
  else if(k == "nstart") to(v, p.nstart, k);
  else if(k == "bc") to(v, p.BC, k);
  else if(k == "no-warning") p.no_warning = true;
  else if(k == "stop-at-warning") p.stop_at_warning = true;
  else if(k == "no-write") p.no_write = true;
  else if(k == "force-delete" || k == "f") p.force_delete = true;
  else if(k == "verbose" || k == "v") to(v.empty() ? string("2") : v, p.verbose, k);
  else if(k == "threads" || k == "t") {}
  else if(k == "save-state") p.save_state = v;
  else return false;
  return true;
}

void set_model_option(const option_list& opts, const string& k, const string& v)
{
  for(const auto& d : opts)
  {
    const int r = d.set_option(k, v);
    if(r == 0) return;
    if(r == -2) throw error_msg("invalid value '", v, "' for option ", k);
  }
  throw error_msg("unknown option '", k, "'");
}

// Files are written by a background thread while the time loop goes on;
// the next write (and the end of the run) waits for the previous one and
// reports its failure.
class AsyncFileWriter
{
  thread worker;
  string failure;

public:
  void wait()
  {
    if(worker.joinable()) worker.join();
    if(!failure.empty())
    {
      const string f = failure;
      failure.clear();
      throw error_msg(f);
    }
  }
  void write(const string& path, string&& text)
  {
    wait();
    worker = thread([this, path](string t) {
      ofstream ofs(path.c_str(), ios::out);
      ofs << t;
      if(!ofs.good()) failure = "can not write " + path;
    }, std::move(text));
  }
  ~AsyncFileWriter() { if(worker.joinable()) worker.join(); }
};

// An output stream buffer that appends to a string (a stringstream copies a
// 74 MB frame at well under 1 GB/s on insertion and once more in str()).
class StringSink : public streambuf
{
public:
  string data;

protected:
  streamsize xsputn(const char* s, streamsize n) override
  {
    data.append(s, static_cast<size_t>(n));
    return n;
  }
  int_type overflow(int_type c) override
  {
    if(c != traits_type::eof()) data.push_back(static_cast<char>(c));
    return c;
  }
};

template<class Writer>
void write_json(AsyncFileWriter& out, const string& path, const string& id, Writer&& w)
{
  StringSink sink;
  {
    ostream os(&sink);
    oarchive ar(os, id, 1);
    w(ar);
    if(ar.bad_value()) throw error_msg("nan found while writing file.");
  }
  out.write(path, std::move(sink.data));
}

int run(int argc, char** argv)
{
  Program p;
  vector<pair<string, string>> cli;
  for(int i = 1; i < argc; ++i)
  {
    string a = argv[i];
    if(a.rfind("--", 0) == 0)
    {
      a = a.substr(2);
      const auto eq = a.find('=');
      if(eq != string::npos) cli.emplace_back(a.substr(0, eq), a.substr(eq + 1));
      else if(i + 1 < argc && argv[i + 1][0] != '-' &&
              a != "no-write" && a != "no-warning" && a != "stop-at-warning" && a != "force-delete")
        cli.emplace_back(a, argv[++i]);
      else cli.emplace_back(a, "");
    }
    else if(a.size() == 2 && a[0] == '-')
    {
      const string k = a.substr(1);
      if((k == "o" || k == "m" || k == "t" || k == "v") && i + 1 < argc) cli.emplace_back(k, argv[++i]);
      else cli.emplace_back(k, "");
    }
    else if(p.inputname.empty()) p.inputname = a;
    else throw error_msg("unexpected argument '", a, "'");
  }
  if(p.inputname.empty()) throw error_msg("please provide an input file.");

  const auto card = read_runcard(p.inputname);
  // program options: runcard first, command line overrides
  for(const auto& kv : card) set_program_option(p, kv.first, kv.second);
  for(const auto& kv : cli) set_program_option(p, kv.first, kv.second);
  if(p.model_name.empty()) throw error_msg("please specify model.");
  if(p.ninfo == 0) throw error_msg("ninfo must be positive.");
  if(p.has_seed) set_seed(p.seed);

  DeclareModels();
  ModelPtr model = NewModel(p.model_name, p.LX, p.LY, p.BC);
  const option_list opts = model->GetOptions();
  for(const auto& kv : card)
    if(!set_program_option(p, kv.first, kv.second)) set_model_option(opts, kv.first, kv.second);
  for(const auto& kv : cli)
    if(!set_program_option(p, kv.first, kv.second)) set_model_option(opts, kv.first, kv.second);
  if(p.nstart % p.ninfo) p.nstart = (1u + p.nstart/p.ninfo)*p.ninfo;

  model->Initialize();
  model->Configure();

  string output_dir = p.runname + (p.runname.back() == '/' ? "" : "/");
  AsyncFileWriter files;
  if(!p.no_write)
  {
    if(system(("mkdir -p '" + output_dir + "'").c_str()) != 0)
      throw error_msg("can not create output directory ", output_dir);
    write_json(files, output_dir + "parameters.json", "parameters", [&](oarchive& ar) {
      unsigned LX = p.LX, LY = p.LY, BC = p.BC, nsteps = p.nsteps, ninfo = p.ninfo,
               nstart = p.nstart, nsubsteps_ = nsubsteps;
      unsigned& nsubsteps = nsubsteps_;
      string model_name = p.model_name;
      ar & auto_name(LX) & auto_name(LY) & auto_name(BC) & auto_name(nsteps)
         & auto_name(nsubsteps) & auto_name(ninfo) & auto_name(nstart)
         & auto_name(model_name);
      model.ptr->serialize_params(ar);
    });
  }

  auto write_frame = [&](unsigned t) {
    write_json(files, output_dir + "frame" + to_string(t) + ".json", "frame",
               [&](oarchive& ar) { model.ptr->serialize_frame(ar); });
  };

  model->Pre();
  model->PreRunStats();
  const auto start = chrono::steady_clock::now();
  for(unsigned t = 0; t < p.nsteps; ++t)
  {
    if(t % p.ninfo == 0)
    {
      if(!p.no_write && t >= p.nstart) write_frame(t);
      if(p.verbose) cout << "timesteps t = " << t << " to " << t + p.ninfo << endl;
    }
    for(unsigned s = 0; s < nsubsteps; ++s) model->Step();
    if(t % p.ninfo == 0 && !p.no_warning)
    {
      try
      {
        if(p.verbose > 1) model->RuntimeStats();
        model->RuntimeChecks();
      }
      catch(const warning_msg& e)
      {
        if(p.stop_at_warning) throw;
        if(p.verbose) cerr << "warning: " << e.what() << endl;
      }
    }
  }
  if(!p.no_write && p.nsteps >= p.nstart) write_frame(p.nsteps);
  files.wait();
  mass_lb_handle* h = nullptr;
  if(auto* l = dynamic_cast<LyotropicGPU*>(model.operator->())) h = l->device_lattice();
  else if(auto* n = dynamic_cast<NematicGPU*>(model.operator->())) h = n->device_lattice();
  // the run time covers the device work the loop queued
  if(h && mass_lb_synchronize(h) != MASS_LB_OK)
    throw error_msg("mass_lb_synchronize: ", mass_lb_last_error());
  const auto dt = chrono::duration<double>(chrono::steady_clock::now() - start).count();
  model->Post();
  if(!p.save_state.empty())
  {
    if(!h) throw error_msg("model '", p.model_name, "' has no device lattice to save");
    if(mass_lb_save(h, p.save_state.c_str()) != MASS_LB_OK)
      throw error_msg("mass_lb_save: ", mass_lb_last_error());
  }
  if(p.verbose) cout << "Total run time :                    " << dt << " s" << endl;
  return 0;
}

} // namespace

int main(int argc, char** argv)
{
  try
  {
    return run(argc, argv);
  }
  catch(const error_msg& e)
  {
    cerr << argv[0] << ": error: " << e.what() << endl;
    return 1;
  }
  catch(const warning_msg& e)
  {
    cerr << argv[0] << ": warning: " << e.what() << endl;
    return 1;
  }
  catch(const exception& e)
  {
    cerr << argv[0] << ": " << e.what() << endl;
    return 1;
  }
}
