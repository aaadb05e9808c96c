// output_queue_check.cpp -- CPU check of the drop-in class's background writer
// (boson_cloud_binary_b200/host/cnm_output_queue.hpp):
//   * jobs run in the order they were posted, on one thread other than the poster's;
//   * drain() returns only after every job posted before it has run;
//   * no more than max_heavy heavy jobs are ever queued or running (post blocks);
//   * a throwing job is reported and the jobs after it still run;
//   * inline mode runs the job before post() returns;
//   * stop() runs what is queued, and a later post() starts a new thread;
// and the snapshot text (host/cnm_snapshot_text.hpp): the same bytes as writing every value
// through an std::ostream, whatever the number of formatting threads.
//
//   output_queue_check        exit status 0 on success
#include <atomic>
#include <chrono>
#include <cstdio>
#include <stdexcept>
#include <thread>
#include <vector>

#include "../boson_cloud_binary_b200/host/cnm_output_queue.hpp"
#include "../boson_cloud_binary_b200/host/cnm_snapshot_text.hpp"

#include <cmath>
#include <complex>
#include <limits>
#include <random>
#include <sstream>
#include <string>

namespace {

int failures = 0;

void require(bool ok, const char *msg)
{
    if (!ok) {
        std::fprintf(stderr, "FAIL: %s\n", msg);
        ++failures;
    }
}

}  // namespace

int main()
{
    const std::thread::id poster = std::this_thread::get_id();
    {  // order, thread, drain
        OutputQueue q;
        std::vector<int> seen;  // touched by the writer thread only until drain()
        std::atomic<bool> other_thread{true};
        for (int k = 0; k < 2000; ++k)
            q.post([&, k] {
                if (std::this_thread::get_id() == poster) other_thread = false;
                seen.push_back(k);
            });
        q.drain();
        require(seen.size() == 2000, "drain returned before every job ran");
        bool ordered = true;
        for (int k = 0; k < (int)seen.size(); ++k) ordered = ordered && seen[(size_t)k] == k;
        require(ordered, "jobs ran out of order");
        require(other_thread.load(), "a job ran on the posting thread");
    }
    {  // heavy jobs are bounded; light ones are not
        OutputQueue q(2);
        std::atomic<int> running{0}, peak{0}, done{0};
        for (int k = 0; k < 12; ++k) {
            q.post(
                [&] {
                    const int r = ++running;
                    int p = peak.load();
                    while (r > p && !peak.compare_exchange_weak(p, r)) {
                    }
                    std::this_thread::sleep_for(std::chrono::milliseconds(2));
                    --running;
                    ++done;
                },
                true);
            require(q.heavy_in_flight() <= 2, "more than two heavy jobs queued");
        }
        q.drain();
        require(done.load() == 12, "heavy jobs lost");
        require(peak.load() == 1, "jobs overlapped (one writer thread)");
        require(q.heavy_in_flight() == 0, "heavy count not released");
    }
    {  // a throwing job does not stop the queue
        OutputQueue q;
        std::atomic<int> after{0};
        q.post([] { throw std::runtime_error("planted failure (expected in this check)"); });
        q.post([&] { ++after; });
        q.drain();
        require(after.load() == 1, "the job after a throwing one did not run");
    }
    {  // inline mode
        OutputQueue q;
        q.inline_mode = true;
        bool ran = false;
        std::thread::id where;
        q.post([&] {
            ran = true;
            where = std::this_thread::get_id();
        });
        require(ran && where == poster, "inline job did not run on the posting thread before post returned");
        q.drain();
    }
    {  // stop runs the queue, a later post restarts the thread
        OutputQueue q;
        std::atomic<int> n{0};
        for (int k = 0; k < 50; ++k) q.post([&] { ++n; });
        q.stop();
        require(n.load() == 50, "stop returned before the queue was empty");
        q.post([&] { ++n; });
        q.drain();
        require(n.load() == 51, "post after stop did not run");
    }
    {  // snapshot text: the bytes of an std::ostream, for 1 to 8 formatting threads
        std::mt19937_64 gen(7);
        std::uniform_real_distribution<double> u(-1.0, 1.0);
        std::vector<std::complex<double>> v(300000);
        for (auto &z : v) z = {u(gen) * std::pow(10.0, (int)(u(gen) * 30)), u(gen) * std::pow(10.0, (int)(u(gen) * 30))};
        const double inf = std::numeric_limits<double>::infinity();
        const double specials[] = {0.0, -0.0, 1.0, -1.0, 1e-300, 5e-324, 123456.5, 1234567.0, 1e-5, inf, -inf,
                                   std::nan(""), 9.999995e-5, -2.5e16};
        for (size_t k = 0; k < sizeof(specials) / sizeof(specials[0]); ++k) v[k] = {specials[k], -specials[k]};
        std::ostringstream ref;
        for (const auto &z : v) ref << z.real() << " " << z.imag() << "\n";
        for (unsigned threads : {1u, 3u, 8u}) {
            std::string all;
            for (const std::string &piece : snapshot_text(v.data(), v.size(), threads)) all += piece;
            require(all == ref.str(), "snapshot text differs from stream formatting");
        }
        std::string none;
        for (const std::string &piece : snapshot_text(v.data(), 0, 4)) none += piece;
        require(none.empty(), "empty snapshot not empty");
    }
    if (failures) return 1;
    std::printf("output_queue_check: OK\n");
    return 0;
}
