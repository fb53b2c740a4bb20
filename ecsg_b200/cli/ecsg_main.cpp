// ecsg_main.cpp -- the reference's command-line driver (main.cpp) on the B200
// library: same key=value parameters, same RSF inputs and outputs, the time
// loop as one fused device run.
//
//   ecsg_main num_grids=2 radius=1 dt=0.589378 imode=1 top_bc=1 check_energy=y
//             movie_dt=17.68 movie_nt=39 movie_vx_flag=y
//             buoy_1=... s11_1=... s13_1=... buoy_2=... s11_2=... s13_2=...
//             src=src.rsf rec_in=rec.rsf rec_out=rec_out.rsf energy_trace=e.rsf
//
// Parameters of main.cpp:36-67, 135-142 with its defaults: num_threads (read,
// not needed), check_energy=n, radius (required; 1 on the device), dt
// (required, ms), imode=1, verb=n, top_bc=0, num_grids=1, movie_dt and
// movie_nt (required), movie_v{x,y,z}_flag=n.  Files (init_del_par_field.cpp,
// init_src.cpp, init_del_rec_trace.cpp): buoy_N, s11_N, s13_N, src, rec_in;
// outputs rec_out, energy_trace (check_energy), res_trace (verb, num_grids > 1),
// movie_v?_N (flags).  Added: precision=f32|f64 (default f32; f64 reproduces
// the reference's double build to its rounding), device=0, graph=y,
// src_comp=0, rec_comp=0, mirror_fix=n, ii_skip_end_column=n, datapath= (write
// samples to separate files there instead of after the header), dryrun=y
// (read the inputs, print the set-up, run nothing), checkpoint=path with
// checkpoint_every=K (write the run state after every K completed steps) and
// stop_after=M (stop after M steps, writing the checkpoint), resume=path
// (continue a checkpointed run: the outputs are those of an uninterrupted run;
// movies cannot be continued).
//
// The loop is main.cpp:165-261: niter = 0 .. ceil(movie_dt*movie_nt/dt).  It
// runs on the device in segments that end at the steps where main.cpp prints
// a movie frame (main.cpp:253-258); each frame is packed on the device, copied
// into a page-locked buffer and written by a host thread while the next
// segment runs.
#include "ecsg_b200.h"
#include "rsf_io.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

using ecsg_cli::RsfIn;
using ecsg_cli::RsfOut;

namespace {

struct Params {
    std::map<std::string, std::string> kv;
    bool has(const std::string &k) const { return kv.count(k) != 0; }
    std::string str(const std::string &k, const std::string &d = "") const
    {
        auto it = kv.find(k);
        return it == kv.end() ? d : it->second;
    }
    int i(const std::string &k, int d) const { return has(k) ? (int)std::strtol(str(k).c_str(), nullptr, 10) : d; }
    double f(const std::string &k, double d) const { return has(k) ? std::strtod(str(k).c_str(), nullptr) : d; }
    // Madagascar booleans: y/Y/1 true, n/N/0 false
    bool b(const std::string &k, bool d) const
    {
        if (!has(k)) return d;
        const std::string v = str(k);
        if (v.empty()) return d;
        return v[0] == 'y' || v[0] == 'Y' || v[0] == '1' || v[0] == 't' || v[0] == 'T';
    }
    std::string file(const std::string &tag) const
    {
        if (!has(tag)) throw std::runtime_error("no file given for '" + tag + "'");
        return str(tag);
    }
};

struct Grid {
    int size[3];
    double step[3];
    double origin[3];
};

[[noreturn]] void die(const std::string &msg)
{
    std::fprintf(stderr, "ecsg_main: %s\n", msg.c_str());
    std::exit(1);
}

void ck(int rc, const char *what, ecsg_sim *sim)
{
    if (rc != ECSG_OK) die(std::string(what) + ": " + (sim ? ecsg_last_error(sim) : "error"));
}

// (grid, ix, iy, iz) of a point as init_src.cpp:33-45 and
// init_del_rec_trace.cpp:31-43 compute it: walk down the grids by depth, then
// round to the nearest node
void locate(const std::vector<Grid> &grids, const double p[3], int loc[4])
{
    int g = 0;
    double z = p[2];
    while (z > grids[g].step[2] * grids[g].size[2]) {
        z -= grids[g].step[2] * grids[g].size[2];
        g++;
        if (g >= (int)grids.size()) die("point below the last grid");
    }
    loc[0] = g;
    for (int d = 0; d < 2; d++) loc[1 + d] = (int)std::lround((p[d] - grids[g].origin[d]) / grids[g].step[d]);
    loc[3] = (int)std::lround(z / grids[g].step[2]);
}

// Frame writer: page-locked buffers filled from the device, written in order
// by one host thread.
class FrameWriter {
public:
    FrameWriter(size_t frame_floats, int nbuf) : floats_(frame_floats)
    {
        for (int b = 0; b < nbuf; b++) {
            void *p = nullptr;
            if (ecsg_host_alloc(frame_floats * sizeof(float), &p) != ECSG_OK) die("page-locked frame buffer");
            free_.push_back((float *)p);
            all_.push_back((float *)p);
        }
        th_ = std::thread([this] { loop(); });
    }
    ~FrameWriter()
    {
        {
            std::lock_guard<std::mutex> l(m_);
            done_ = true;
        }
        cv_.notify_all();
        th_.join();
        for (float *p : all_) ecsg_host_free(p);
    }
    float *acquire()
    {
        std::unique_lock<std::mutex> l(m_);
        cv_.wait(l, [this] { return !free_.empty() || !error_.empty(); });
        if (!error_.empty()) die(error_);
        float *p = free_.front();
        free_.pop_front();
        return p;
    }
    void submit(RsfOut *out, float *buf, size_t n)
    {
        {
            std::lock_guard<std::mutex> l(m_);
            jobs_.push_back({out, buf, n});
        }
        cv_.notify_all();
    }
    void drain()
    {
        std::unique_lock<std::mutex> l(m_);
        cv_.wait(l, [this] { return (jobs_.empty() && free_.size() == all_.size()) || !error_.empty(); });
        if (!error_.empty()) die(error_);
    }

private:
    struct Job {
        RsfOut *out;
        float *buf;
        size_t n;
    };
    void loop()
    {
        for (;;) {
            Job j;
            {
                std::unique_lock<std::mutex> l(m_);
                cv_.wait(l, [this] { return !jobs_.empty() || done_; });
                if (jobs_.empty()) return;
                j = jobs_.front();
                jobs_.pop_front();
            }
            try {
                j.out->write(j.buf, j.n);
            } catch (const std::exception &e) {
                std::lock_guard<std::mutex> l(m_);
                error_ = e.what();
            }
            {
                std::lock_guard<std::mutex> l(m_);
                free_.push_back(j.buf);
            }
            cv_.notify_all();
        }
    }
    size_t floats_;
    std::vector<float *> all_;
    std::deque<float *> free_;
    std::deque<Job> jobs_;
    std::mutex m_;
    std::condition_variable cv_;
    std::thread th_;
    bool done_ = false;
    std::string error_;
};

// Checkpoint file: an RSF-style header (the set-up it belongs to, the number
// of completed steps, the sizes of the parts), then 0x0c 0x0c 0x04, the
// library's run state (ecsg_save_state), the receiver samples, energies and
// residues of the completed steps.
void write_checkpoint(const std::string &path, const std::string &setup, int done, long long state_bytes,
                      ecsg_sim *sim, const std::vector<float> &rec, const std::vector<double> &energy,
                      const std::vector<double> &res)
{
    const std::string tmp = path + ".partial";
    FILE *fp = std::fopen(tmp.c_str(), "wb");
    if (!fp) die("cannot create " + tmp);
    std::vector<unsigned char> state((size_t)state_bytes);
    ck(ecsg_save_state(sim, state.data()), "ecsg_save_state", sim);
    std::fprintf(fp, "ecsg_checkpoint=1 %s done=%d state_bytes=%lld\n", setup.c_str(), done, state_bytes);
    std::fputc(0x0c, fp);
    std::fputc(0x0c, fp);
    std::fputc(0x04, fp);
    bool ok = std::fwrite(state.data(), 1, state.size(), fp) == state.size();
    // histories: the whole arrays (steps after `done` are unset and ignored on resume)
    ok = ok && std::fwrite(rec.data(), sizeof(float), rec.size(), fp) == rec.size();
    ok = ok && std::fwrite(energy.data(), sizeof(double), energy.size(), fp) == energy.size();
    ok = ok && std::fwrite(res.data(), sizeof(double), res.size(), fp) == res.size();
    ok = (std::fclose(fp) == 0) && ok;
    if (!ok || std::rename(tmp.c_str(), path.c_str()) != 0) die("cannot write checkpoint " + path);
}

int read_checkpoint(const std::string &path, const std::string &setup, long long state_bytes, ecsg_sim *sim,
                    std::vector<float> &rec, std::vector<double> &energy, std::vector<double> &res)
{
    FILE *fp = std::fopen(path.c_str(), "rb");
    if (!fp) die("cannot open checkpoint " + path);
    std::string text;
    int c, p1 = -1, p2 = -1;
    bool marker = false;
    while ((c = std::fgetc(fp)) != EOF) {
        if (p2 == 0x0c && p1 == 0x0c && c == 0x04) { marker = true; text.resize(text.size() - 2); break; }
        text.push_back((char)c);
        p2 = p1;
        p1 = c;
    }
    if (!marker) die(path + ": not a checkpoint");
    std::map<std::string, std::string> kv, want;
    ecsg_cli::parse_pairs(text, kv);
    ecsg_cli::parse_pairs(setup, want);
    if (kv["ecsg_checkpoint"] != "1") die(path + ": not a checkpoint");
    for (auto &w : want)
        if (kv[w.first] != w.second)
            die(path + ": written for " + w.first + "=" + kv[w.first] + ", this run has " + w.second);
    if (std::strtoll(kv["state_bytes"].c_str(), nullptr, 10) != state_bytes) die(path + ": state size differs");
    const int done = (int)std::strtol(kv["done"].c_str(), nullptr, 10);
    std::vector<unsigned char> state((size_t)state_bytes);
    bool ok = std::fread(state.data(), 1, state.size(), fp) == state.size();
    ok = ok && std::fread(rec.data(), sizeof(float), rec.size(), fp) == rec.size();
    ok = ok && std::fread(energy.data(), sizeof(double), energy.size(), fp) == energy.size();
    ok = ok && std::fread(res.data(), sizeof(double), res.size(), fp) == res.size();
    std::fclose(fp);
    if (!ok || done <= 0) die(path + ": truncated checkpoint");
    ck(ecsg_load_state(sim, state.data()), "ecsg_load_state", sim);
    return done;
}

int run(const Params &P)
{
    const bool check_energy = P.b("check_energy", false);
    const int radius = P.i("radius", 0);
    const double dt = P.f("dt", -1.0);
    const int imode = P.i("imode", 1);
    const bool verb = P.b("verb", false);
    const int top_bc = P.i("top_bc", 0);
    const int num_grids = P.i("num_grids", 1);
    const double movie_dt = P.f("movie_dt", -1.0);
    const int movie_nt = P.i("movie_nt", -1);
    const bool movie_flag[3] = {P.b("movie_vx_flag", false), P.b("movie_vy_flag", false), P.b("movie_vz_flag", false)};
    const std::string precision = P.str("precision", "f32");
    const std::string datapath = P.str("datapath", "");
    if (radius <= 0) die("radius must be given (> 0)");
    if (!(dt > 0)) die("dt must be given (> 0, ms)");
    if (!(movie_dt > 0) || movie_nt <= 0) die("movie_dt and movie_nt must be given (> 0)");
    if (num_grids < 1) die("num_grids must be >= 1");
    if (precision != "f32" && precision != "f64") die("precision must be f32 or f64");

    // grids and media (init_del_par_field.cpp:22-76, 91-117)
    std::vector<Grid> grids(num_grids);
    std::vector<std::vector<float>> media(3 * num_grids);
    const char *med_tag[3] = {"buoy_", "s11_", "s13_"};
    for (int g = 0; g < num_grids; g++) {
        for (int m = 0; m < 3; m++) {
            const std::string tag = med_tag[m] + std::to_string(g + 1);
            RsfIn in(P.file(tag));
            int n[3];
            for (int d = 0; d < 3; d++) {
                n[d] = in.get_int("n" + std::to_string(d + 1), -1) - 1;
                const double h = in.get_double("d" + std::to_string(d + 1), -1.0);
                if (n[d] <= 0 || !(h > 0)) die(tag + ": n1..n3 must be > 1 and d1..d3 > 0");
                if (m == 0) {
                    grids[g].size[d] = n[d];
                    grids[g].step[d] = h;
                } else if (n[d] != grids[g].size[d]) {
                    die(tag + ": size differs from buoy_" + std::to_string(g + 1));
                }
            }
            media[3 * g + m] = in.read((size_t)(n[0] + 1) * (n[1] + 1) * (n[2] + 1));
        }
        grids[g].origin[0] = grids[g].origin[1] = 0.0;
        grids[g].origin[2] = g == 0 ? 0.0 : grids[g - 1].origin[2] + grids[g - 1].size[2] * grids[g - 1].step[2];
    }

    // source (init_src.cpp:7-49): n1 samples; its position in o2, o3, o4
    RsfIn src(P.file("src"));
    const int src_nt = src.get_int("n1", 0);
    std::vector<float> src_trace = src.read((size_t)(src_nt > 0 ? src_nt : 0));
    const double src_xyz[3] = {src.get_double("o2", 0.0), src.get_double("o3", 0.0), src.get_double("o4", 0.0)};
    int src_loc[4];
    locate(grids, src_xyz, src_loc);
    std::printf("== Source is placed at... \n(grid#%d, ix=%d, iy=%d, iz=%d)\n", src_loc[0], src_loc[1], src_loc[2],
                src_loc[3]);

    // receivers (init_del_rec_trace.cpp:8-56): n2 points of 3 floats
    RsfIn rec_in(P.file("rec_in"));
    const int n_rec = rec_in.get_int("n2", 0);
    std::vector<int> rec_loc(4 * (size_t)n_rec);
    std::printf("== Record traces at... \n");
    for (int r = 0; r < n_rec; r++) {
        float p[3];
        rec_in.read(p, 3);
        const double pd[3] = {p[0], p[1], p[2]};
        locate(grids, pd, &rec_loc[4 * r]);
        std::printf("(grid#%d, ix=%d,  iy=%d, iz=%d)\n", rec_loc[4 * r], rec_loc[4 * r + 1], rec_loc[4 * r + 2],
                    rec_loc[4 * r + 3]);
    }

    // steps and movie frames (main.cpp:165, 253-258)
    const int last = (int)std::ceil(movie_dt * movie_nt / dt);
    const int nsteps = last + 1;
    std::vector<int> frame_steps;
    for (int niter = 0, iframe = 0; niter <= last; niter++)
        if (iframe < movie_nt && niter * dt <= iframe * movie_dt && iframe * movie_dt < niter * dt + dt) {
            frame_steps.push_back(niter);
            iframe++;
        }
    std::fflush(stdout);
    if (P.b("dryrun", false)) {
        std::printf("== Grids\n");
        for (int g = 0; g < num_grids; g++)
            std::printf("grid_%d size %d %d %d step %.9g %.9g %.9g origin %.9g %.9g %.9g\n", g + 1, grids[g].size[0],
                        grids[g].size[1], grids[g].size[2], grids[g].step[0], grids[g].step[1], grids[g].step[2],
                        grids[g].origin[0], grids[g].origin[1], grids[g].origin[2]);
        std::printf("== Steps %d, frames %zu:", nsteps, frame_steps.size());
        for (int s : frame_steps) std::printf(" %d", s);
        std::printf("\n");
        return 0;
    }

    // device state
    std::vector<ecsg_grid_desc> gd(num_grids);
    for (int g = 0; g < num_grids; g++)
        for (int d = 0; d < 3; d++) {
            gd[g].size[d] = grids[g].size[d];
            gd[g].step[d] = grids[g].step[d];
        }
    ecsg_config cfg = {num_grids, radius, dt, imode, top_bc, precision == "f64" ? ECSG_F64 : ECSG_F32,
                       ECSG_MEDIUM_ISO, check_energy ? 1 : 0, 0, P.i("device", 0), P.b("mirror_fix", false) ? 1 : 0,
                       P.b("ii_skip_end_column", false) ? 1 : 0};
    ecsg_sim *sim = nullptr;
    ck(ecsg_create(gd.data(), &cfg, &sim), "ecsg_create", sim);
    for (int g = 0; g < num_grids; g++)
        ck(ecsg_set_medium_iso(sim, g, media[3 * g].data(), media[3 * g + 1].data(), media[3 * g + 2].data()),
           "ecsg_set_medium_iso", sim);
    media.clear();
    media.shrink_to_fit();
    if (src_nt > 0)
        ck(ecsg_set_source(sim, src_loc[0], src_loc[1], src_loc[2], src_loc[3], P.i("src_comp", 0), src_trace.data(),
                           src_nt, 1000.0f),
           "ecsg_set_source", sim);
    ck(ecsg_set_receivers(sim, rec_loc.data(), n_rec, P.i("rec_comp", 0)), "ecsg_set_receivers", sim);

    // movies (init_del_movie.cpp:5-54): header first, one frame per print
    std::vector<std::unique_ptr<RsfOut>> movies;
    std::vector<std::pair<int, int>> movie_src;   // (grid, component)
    size_t max_frame = 0;
    const char *vname[3] = {"vx", "vy", "vz"};
    for (int j = 0; j < 3; j++)
        if (movie_flag[j])
            for (int g = 0; g < num_grids; g++) {
                const std::string tag = std::string("movie_") + vname[j] + "_" + std::to_string(g + 1);
                int dims[3];
                ck(ecsg_domain_shape(sim, g, j, dims), "ecsg_domain_shape", sim);
                auto out = std::make_unique<RsfOut>(P.file(tag), datapath);
                for (int d = 0; d < 3; d++) out->put("n" + std::to_string(d + 1), dims[d]);
                out->put("n4", movie_nt);
                for (int d = 0; d < 3; d++) out->put("d" + std::to_string(d + 1), (float)grids[g].step[d]);
                out->put("d4", (float)movie_dt);
                for (int d = 0; d < 3; d++) out->put("o" + std::to_string(d + 1), (float)grids[g].origin[d]);
                out->put("o4", 0.0f);
                const char *lab[4] = {"X", "Y", "Z", "Time"}, *unit[4] = {"m", "m", "m", "ms"};
                for (int d = 0; d < 4; d++) {
                    out->put("label" + std::to_string(d + 1), std::string(lab[d]));
                    out->put("unit" + std::to_string(d + 1), std::string(unit[d]));
                }
                max_frame = std::max(max_frame, (size_t)dims[0] * dims[1] * dims[2]);
                movies.push_back(std::move(out));
                movie_src.emplace_back(g, j);
            }
    std::unique_ptr<FrameWriter> writer;
    if (!movies.empty()) writer = std::make_unique<FrameWriter>(max_frame, 2 * (int)movies.size());

    // the loop, in segments ending at frame steps and checkpoint steps
    const bool residues = verb && num_grids > 1;
    std::vector<float> rec((size_t)nsteps * n_rec);
    std::vector<double> energy(check_energy ? nsteps : 0);
    std::vector<double> res(residues ? (size_t)nsteps * (num_grids - 1) * 9 : 0);
    const int use_graph = P.b("graph", true) ? 1 : 0;
    const std::string ckpt_path = P.str("checkpoint", "");
    const int ckpt_every = P.i("checkpoint_every", 0);
    const int stop_after = P.i("stop_after", 0);
    // the set-up a checkpoint must match (key=value, compared as text on resume)
    std::string setup = "num_grids=" + std::to_string(num_grids) + " radius=" + std::to_string(radius) +
                        " imode=" + std::to_string(imode) + " top_bc=" + std::to_string(top_bc) + " precision=" +
                        precision + " check_energy=" + std::to_string((int)check_energy) +
                        " residues=" + std::to_string((int)residues) + " n_rec=" + std::to_string(n_rec) +
                        " nsteps=" + std::to_string(nsteps);
    for (int g = 0; g < num_grids; g++)
        setup += " grid_" + std::to_string(g + 1) + "=" + std::to_string(grids[g].size[0]) + "x" +
                 std::to_string(grids[g].size[1]) + "x" + std::to_string(grids[g].size[2]);
    {
        char buf[64];
        std::snprintf(buf, sizeof buf, " dt=%.17g", dt);
        setup += buf;
    }
    const long long state_bytes = ecsg_state_bytes(sim);
    int start = 0;
    if (P.has("resume")) {
        if (!movies.empty()) die("resume: movies cannot be continued; run without movie flags");
        start = read_checkpoint(P.str("resume"), setup, state_bytes, sim, rec, energy, res);
        std::printf("== Resumed after step %d of %d\n", start - 1, nsteps - 1);
    }
    const int stop = stop_after > 0 && stop_after < nsteps ? stop_after : nsteps;
    const auto t0 = std::chrono::steady_clock::now();
    double device_ms = 0.0;
    size_t next_frame = 0;
    while (next_frame < frame_steps.size() && frame_steps[next_frame] < start) next_frame++;
    for (int n0 = start; n0 < stop;) {
        int end = next_frame < frame_steps.size() ? frame_steps[next_frame] + 1 : stop;
        if (ckpt_every > 0) end = std::min(end, (n0 / ckpt_every + 1) * ckpt_every);
        end = std::min(end, stop);
        const int len = end - n0;
        ck(ecsg_run(sim, n0, len, n_rec ? &rec[(size_t)n0 * n_rec] : nullptr, check_energy ? &energy[n0] : nullptr,
                    1, residues ? &res[(size_t)n0 * (num_grids - 1) * 9] : nullptr, use_graph),
           "ecsg_run", sim);
        double ms = 0.0;
        ecsg_last_run(sim, &ms, nullptr);
        device_ms += ms;
        if (verb)
            for (int n = n0; n < end; n++) std::fprintf(stderr, "niter = %d\n", n);
        if (next_frame < frame_steps.size() && end - 1 == frame_steps[next_frame]) {
            for (size_t m = 0; m < movies.size(); m++) {
                float *buf = writer->acquire();
                int dims[3];
                ecsg_domain_shape(sim, movie_src[m].first, movie_src[m].second, dims);
                ck(ecsg_get_domain(sim, movie_src[m].first, movie_src[m].second, buf), "ecsg_get_domain", sim);
                writer->submit(movies[m].get(), buf, (size_t)dims[0] * dims[1] * dims[2]);
            }
            next_frame++;
        }
        if (!ckpt_path.empty() && ((ckpt_every > 0 && end % ckpt_every == 0) || end == stop) && end < nsteps)
            write_checkpoint(ckpt_path, setup, end, state_bytes, sim, rec, energy, res);
        n0 = end;
    }
    if (stop < nsteps) {
        if (writer) writer->drain();
        std::printf("== Stopped after step %d of %d%s\n", stop - 1, nsteps - 1,
                    ckpt_path.empty() ? "" : (", checkpoint " + ckpt_path).c_str());
        movies.clear();
        writer.reset();
        ecsg_destroy(sim);
        return 0;
    }
    if (writer) writer->drain();
    int status = 0;
    ecsg_get_status(sim, &status, 0);
    const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::printf("Total elapsed time %g s.\n", wall);
    std::printf("Device time of the time loop %g s.\n", device_ms * 1e-3);
    if (status) std::fprintf(stderr, "ecsg_main: device status %d (see include/ecsg_b200.h)\n", status);

    // outputs (print.cpp:29-49, 108-130; main.cpp:275-300)
    if (check_energy) {
        RsfOut out(P.file("energy_trace"), datapath);
        out.put("n1", nsteps);
        out.put("o1", 0.0f);
        out.put("d1", (float)dt);
        out.put("label1", std::string("Time"));
        out.put("unit1", std::string("ms"));
        out.put("n2", 1);
        out.put("n3", 1);
        out.put("n4", 1);
        std::vector<float> e(nsteps);
        for (int n = 0; n < nsteps; n++) e[n] = (float)energy[n];
        out.write(e.data(), e.size());
    }
    {
        RsfOut out(P.file("rec_out"), datapath);
        out.put("n1", nsteps);
        out.put("o1", 0.0f);
        out.put("d1", (float)dt);
        out.put("label1", std::string("Time"));
        out.put("unit1", std::string("ms"));
        out.put("n2", n_rec);
        std::vector<float> tr(nsteps);
        for (int r = 0; r < n_rec; r++) {
            for (int n = 0; n < nsteps; n++) tr[n] = rec[(size_t)n * n_rec + r];
            out.write(tr.data(), tr.size());
        }
    }
    if (residues) {
        RsfOut out(P.file("res_trace"), datapath);
        out.put("n1", nsteps);
        out.put("n2", 9);
        out.put("n3", num_grids - 1);
        std::vector<float> tr(nsteps);
        for (int i = 0; i < num_grids - 1; i++)
            for (int j = 0; j < 9; j++) {
                for (int n = 0; n < nsteps; n++) tr[n] = (float)res[((size_t)n * (num_grids - 1) + i) * 9 + j];
                out.write(tr.data(), tr.size());
            }
    }
    movies.clear();
    writer.reset();
    ecsg_destroy(sim);
    return status ? 3 : 0;
}

} // namespace

int main(int argc, char **argv)
{
    Params P;
    for (int i = 1; i < argc; i++) {   // key=value per argument (sf_init); later ones win
        const std::string a(argv[i]);
        const size_t eq = a.find('=');
        if (eq == std::string::npos || eq == 0) continue;
        std::string v = a.substr(eq + 1);
        if (v.size() >= 2 && v.front() == '"' && v.back() == '"') v = v.substr(1, v.size() - 2);
        P.kv[a.substr(0, eq)] = v;
    }
    try {
        return run(P);
    } catch (const std::exception &e) {
        die(e.what());
    }
}
