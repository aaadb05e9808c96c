// cnm_output_queue.hpp -- the drop-in class's background writer.
//
// The reference formats every diagnostic row and every state snapshot on the stepping
// thread (src/CrankNicolsonModes_utils.cpp:48-83): a snapshot of 153 modes x 65536 nodes
// is 10 M text lines, seconds of formatting for a step of milliseconds.  Here the stepping
// thread only copies the state off the device; the rows, snapshots and checkpoint files are
// written by one background thread that runs the posted jobs in the order they were posted,
// so every file receives exactly the bytes, in the same order, that synchronous writing
// would give it (and a checkpoint is still renamed into place only after the snapshot and
// the diagnostic rows before it are written).
//
// Heavy jobs (snapshots) are bounded: post() blocks while `max_heavy` of them are queued or
// running, so a writer slower than the solver holds back the solver instead of the memory.
// drain() returns once every job posted before it has run.  A job that throws has its
// message printed to stderr, as the reference does for a file it cannot open, and the
// queue carries on.
#pragma once

#include <condition_variable>
#include <cstddef>
#include <deque>
#include <exception>
#include <functional>
#include <iostream>
#include <mutex>
#include <thread>
#include <utility>

class OutputQueue {
public:
    explicit OutputQueue(size_t max_heavy = 2) : max_heavy_(max_heavy < 1 ? 1 : max_heavy) {}
    ~OutputQueue() { stop(); }
    OutputQueue(const OutputQueue &) = delete;
    OutputQueue &operator=(const OutputQueue &) = delete;

    /// Queue `job` behind every job posted so far (runs it inline when `inline_mode` is set).
    void post(std::function<void()> job, bool heavy = false)
    {
        if (inline_mode) {
            run_one(job);
            return;
        }
        std::unique_lock<std::mutex> lk(m_);
        if (!thread_.joinable()) thread_ = std::thread([this] { loop(); });
        if (heavy) {
            room_.wait(lk, [this] { return heavy_ < max_heavy_; });
            ++heavy_;
        }
        jobs_.emplace_back(std::move(job), heavy);
        ++posted_;
        work_.notify_one();
    }

    /// Wait until every job posted so far has run.
    void drain()
    {
        std::unique_lock<std::mutex> lk(m_);
        const unsigned long long target = posted_;
        done_.wait(lk, [&] { return finished_ >= target; });
    }

    /// Drain and end the background thread (post() starts a new one).
    void stop()
    {
        {
            std::unique_lock<std::mutex> lk(m_);
            if (!thread_.joinable()) return;
            quit_ = true;
            work_.notify_one();
        }
        thread_.join();
        std::lock_guard<std::mutex> lk(m_);
        quit_ = false;
    }

    /// Heavy jobs queued or running (for tests).
    size_t heavy_in_flight()
    {
        std::lock_guard<std::mutex> lk(m_);
        return heavy_;
    }

    /// Run every job on the posting thread instead (synchronous writing).
    bool inline_mode = false;

private:
    std::mutex m_;
    std::condition_variable work_, done_, room_;
    std::deque<std::pair<std::function<void()>, bool>> jobs_;
    std::thread thread_;
    size_t max_heavy_, heavy_ = 0;
    unsigned long long posted_ = 0, finished_ = 0;
    bool quit_ = false;

    static void run_one(std::function<void()> &job)
    {
        try {
            job();
        } catch (const std::exception &e) {
            std::cerr << "output writer: " << e.what() << "\n";
        } catch (...) {
            std::cerr << "output writer: unknown error\n";
        }
    }

    void loop()
    {
        for (;;) {
            std::pair<std::function<void()>, bool> item;
            {
                std::unique_lock<std::mutex> lk(m_);
                work_.wait(lk, [this] { return quit_ || !jobs_.empty(); });
                if (jobs_.empty()) return;  // quit_ with nothing left: every job has run
                item = std::move(jobs_.front());
                jobs_.pop_front();
            }
            run_one(item.first);
            item.first = nullptr;  // release the job's buffers before it counts as finished
            std::lock_guard<std::mutex> lk(m_);
            ++finished_;
            if (item.second) {
                --heavy_;
                room_.notify_all();
            }
            done_.notify_all();
        }
    }
};
