// harmony_serve — the reference's TCP serving path over libhy.so on one GPU.
//
// The reference serves queries from its MPI master: an optional INSERT phase
// on a first connection (src/query.cpp:24-32 opcodes, 486-656), then a query
// server (src/master_server.h:5-8, src/master_server.cpp:106-199) that reads
// [uint64 nq][uint64 k][nq*d float32] and answers
// [nq*k float32 distances][nq*k int64 labels]; nq = 0 ends the server.  The
// protocol here is the same, little-endian, byte for byte, so the reference's
// unmodified harmony_client (src/client.cpp) talks to it.  Each query batch
// is one hy_index_search call (in graph mode, batches of a repeated shape
// replay a captured CUDA graph).
//
//   harmony_serve --index FILE [--port 7777] [common options]
//       load a .index file (the reference's --skip_insert --cache path)
//   harmony_serve --train_data FILE.fvecs [--nlist N] [--insert_port P] [--save FILE]
//                 [--port 7777] [common options]
//       train on the seed file, then take OP_INSERT batches and OP_BUILD_DONE
//       on the insert port (add + preSearch), then serve queries on --port
//   common: --nprobe N (64) --form plain|bf16|fp8 --graph 0|1 (1)
//           --warmup_list N (10) --warmup_list_size N (0: k) --metric l2|ip
//           --device N
//
// INSERT phase (one client):
//   [uint8 1][uint64 n][n*d float32] -> [uint8 status]   append n vectors
//   [uint8 2]                        -> [uint8 status]   add all, preSearch
//   [uint8 0]                                            abort
// status 0 = OK, 1 = error.  After the BUILD_DONE reply the insert socket is
// closed and the query server listens (the client reconnects), as in the
// reference.
#include <arpa/inet.h>
#include <netinet/in.h>
#include <netinet/tcp.h>
#include <sys/socket.h>
#include <unistd.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/hy.h"

namespace {

constexpr uint8_t OP_SHUTDOWN = 0x00, OP_INSERT = 0x01, OP_BUILD_DONE = 0x02;
constexpr uint8_t STATUS_OK = 0x00, STATUS_ERROR = 0x01;

struct Options {
    std::string index, train_data, save;
    int port = 7777, insert_port = -1, device = 0;
    size_t nlist = 0, nprobe = 64, warmup_list = 10, warmup_list_size = 0;
    int form = HY_FORM_PLAIN, graph = 1, metric = HY_METRIC_L2;
};

[[noreturn]] void die(const std::string& msg) {
    std::fprintf(stderr, "[harmony_serve] %s\n", msg.c_str());
    std::exit(1);
}

void check(int rc, const char* what) {
    if (rc != HY_OK) die(std::string(what) + ": " + hy_last_error());
}

Options parse(int argc, char** argv) {
    Options o;
    std::map<std::string, std::string> kv;
    for (int i = 1; i < argc; ++i) {
        std::string a = argv[i];
        if (a.rfind("--", 0) != 0 || i + 1 >= argc) die("arguments are --name value pairs (at " + a + ")");
        kv[a.substr(2)] = argv[++i];
    }
    auto num = [&](const char* k, size_t def) { return kv.count(k) ? std::stoull(kv[k]) : def; };
    o.index = kv.count("index") ? kv["index"] : "";
    o.train_data = kv.count("train_data") ? kv["train_data"] : "";
    o.save = kv.count("save") ? kv["save"] : "";
    o.port = static_cast<int>(num("port", 7777));
    o.insert_port = static_cast<int>(num("insert_port", static_cast<size_t>(o.port)));
    o.device = static_cast<int>(num("device", 0));
    o.nlist = num("nlist", 0);
    o.nprobe = num("nprobe", 64);
    o.warmup_list = num("warmup_list", 10);
    o.warmup_list_size = num("warmup_list_size", 0);
    o.graph = static_cast<int>(num("graph", 1));
    if (kv.count("form")) {
        const std::string f = kv["form"];
        o.form = f == "plain" ? HY_FORM_PLAIN : f == "bf16" ? HY_FORM_BF16 : f == "fp8" ? HY_FORM_FP8 : -1;
        if (o.form < 0) die("--form must be plain, bf16 or fp8");
    }
    if (kv.count("metric")) {
        const std::string m = kv["metric"];
        o.metric = m == "l2" ? HY_METRIC_L2 : m == "ip" ? HY_METRIC_IP : -1;
        if (o.metric < 0) die("--metric must be l2 or ip");
    }
    if (o.index.empty() == o.train_data.empty()) die("give exactly one of --index FILE and --train_data FILE");
    return o;
}

// [int32 d][d float32] records (the seed file of the insert mode).
std::vector<float> read_fvecs(const std::string& path, size_t* n, size_t* d) {
    std::ifstream in(path, std::ios::binary);
    if (!in) die("cannot open " + path);
    int32_t dd = 0;
    in.read(reinterpret_cast<char*>(&dd), 4);
    if (!in || dd <= 0) die(path + ": not an .fvecs file");
    in.seekg(0, std::ios::end);
    const size_t bytes = static_cast<size_t>(in.tellg());
    const size_t rec = 4 + 4 * static_cast<size_t>(dd);
    *d = static_cast<size_t>(dd);
    *n = bytes / rec;
    std::vector<float> out(*n * *d);
    in.seekg(0);
    std::vector<char> buf(rec);
    for (size_t i = 0; i < *n; ++i) {
        in.read(buf.data(), static_cast<std::streamsize>(rec));
        std::memcpy(&out[i * *d], buf.data() + 4, *d * 4);
    }
    return out;
}

bool send_all(int fd, const void* buf, size_t n) {
    const char* p = static_cast<const char*>(buf);
    while (n > 0) {
        const ssize_t s = ::send(fd, p, n, MSG_NOSIGNAL);
        if (s <= 0) return false;
        p += s;
        n -= static_cast<size_t>(s);
    }
    return true;
}

bool recv_all(int fd, void* buf, size_t n) {
    char* p = static_cast<char*>(buf);
    while (n > 0) {
        const ssize_t s = ::recv(fd, p, n, 0);
        if (s <= 0) return false;
        p += s;
        n -= static_cast<size_t>(s);
    }
    return true;
}

int listen_on(int port) {
    const int fd = ::socket(AF_INET, SOCK_STREAM, 0);
    if (fd < 0) die("socket() failed");
    int one = 1;
    setsockopt(fd, SOL_SOCKET, SO_REUSEADDR, &one, sizeof(one));
    sockaddr_in addr{};
    addr.sin_family = AF_INET;
    addr.sin_addr.s_addr = INADDR_ANY;
    addr.sin_port = htons(static_cast<uint16_t>(port));
    if (::bind(fd, reinterpret_cast<sockaddr*>(&addr), sizeof(addr)) < 0)
        die("bind() failed on port " + std::to_string(port));
    if (::listen(fd, 1) < 0) die("listen() failed");
    return fd;
}

int accept_one(int server) {
    sockaddr_in ca{};
    socklen_t cl = sizeof(ca);
    const int fd = ::accept(server, reinterpret_cast<sockaddr*>(&ca), &cl);
    if (fd < 0) die("accept() failed");
    int one = 1;
    setsockopt(fd, IPPROTO_TCP, TCP_NODELAY, &one, sizeof(one));
    return fd;
}

// INSERT phase: returns once BUILD_DONE has been answered (the index holds
// the inserted vectors and its warm-up parameters), or exits on abort.
void insert_phase(hy_index* h, const Options& o, size_t d) {
    const int server = listen_on(o.insert_port);
    std::printf("[harmony_serve] insert server listening on port %d\n", o.insert_port);
    std::fflush(stdout);
    const int fd = accept_one(server);
    std::vector<float> all;
    for (;;) {
        uint8_t op = OP_SHUTDOWN;
        if (!recv_all(fd, &op, 1) || op == OP_SHUTDOWN) die("insert client left before BUILD_DONE");
        if (op == OP_INSERT) {
            uint64_t n = 0;
            if (!recv_all(fd, &n, sizeof(n))) die("insert client left");
            const size_t old = all.size();
            all.resize(old + static_cast<size_t>(n) * d);
            const bool ok = recv_all(fd, all.data() + old, static_cast<size_t>(n) * d * sizeof(float));
            if (!ok) die("insert client left while sending vectors");
            send_all(fd, &STATUS_OK, 1);
        } else if (op == OP_BUILD_DONE) {
            const size_t n = all.size() / d;
            int rc = hy_index_add(h, n, all.data());
            if (rc == HY_OK && !o.save.empty()) rc = hy_index_save(h, o.save.c_str());
            if (rc == HY_OK) rc = hy_index_presearch(h, o.warmup_list, o.warmup_list_size);
            if (rc != HY_OK) std::fprintf(stderr, "[harmony_serve] build failed: %s\n", hy_last_error());
            std::printf("[harmony_serve] built the lists of %zu vectors\n", n);
            std::fflush(stdout);
            send_all(fd, rc == HY_OK ? &STATUS_OK : &STATUS_ERROR, 1);
            if (rc != HY_OK) die("build failed");
            break;
        } else {
            send_all(fd, &STATUS_ERROR, 1);
        }
    }
    ::close(fd);
    ::close(server);
}

// Query phase (src/master_server.cpp:106-199): one client at a time; a
// header with nq = 0 ends the server.
void query_phase(hy_index* h, const Options& o, size_t d) {
    const int server = listen_on(o.port);
    std::printf("[harmony_serve] query server listening on port %d\n", o.port);
    std::fflush(stdout);
    std::vector<float> q, D;
    std::vector<int64_t> I;
    for (bool stop = false; !stop;) {
        const int fd = accept_one(server);
        for (;;) {
            uint64_t hdr[2] = {0, 0};
            if (!recv_all(fd, hdr, sizeof(hdr))) break;  // client left
            const size_t nq = static_cast<size_t>(hdr[0]), k = static_cast<size_t>(hdr[1]);
            if (nq == 0) {
                stop = true;
                break;
            }
            q.resize(nq * d);
            if (!recv_all(fd, q.data(), q.size() * sizeof(float))) break;
            D.assign(nq * k, 0.0f);
            I.assign(nq * k, -1);
            const int rc = hy_index_search(h, nq, q.data(), k, D.data(), I.data());
            if (rc != HY_OK) {
                // The protocol has no error reply: the connection is closed.
                std::fprintf(stderr, "[harmony_serve] search of %zu queries (k %zu) failed: %s\n", nq, k,
                             hy_last_error());
                break;
            }
            if (!send_all(fd, D.data(), D.size() * sizeof(float)) ||
                !send_all(fd, I.data(), I.size() * sizeof(int64_t)))
                break;
        }
        ::close(fd);
    }
    ::close(server);
}

}  // namespace

int main(int argc, char** argv) {
    const Options o = parse(argc, argv);
    hy_index* h = nullptr;
    size_t d = 0;
    if (!o.index.empty()) {
        size_t nlist = 0, nonempty = 0, ntotal = 0;
        int metric = 0, opt = 0;
        check(hy_file_inspect(o.index.c_str(), &d, &nlist, &metric, &opt, &nonempty, &ntotal), "inspect index");
        check(hy_index_create(d, nlist, o.nprobe, metric, 0, 0, o.device, &h), "create");
        check(hy_index_load(h, o.index.c_str()), "load");
        check(hy_index_presearch(h, o.warmup_list, o.warmup_list_size), "presearch");
        std::printf("[harmony_serve] loaded %zu vectors, d %zu, %zu lists\n", ntotal, d, nlist);
    } else {
        size_t n = 0;
        std::vector<float> seed = read_fvecs(o.train_data, &n, &d);
        size_t nlist = o.nlist;
        if (nlist == 0) {
            nlist = 1;
            while ((nlist + 1) * (nlist + 1) <= n) ++nlist;  // sqrt(n), as the reference picks it
        }
        check(hy_index_create(d, nlist, o.nprobe, o.metric, 0, 0, o.device, &h), "create");
        check(hy_index_train(h, n, seed.data(), 0), "train");
        std::printf("[harmony_serve] trained %zu lists on %zu seed vectors (d %zu)\n", nlist, n, d);
    }
    std::fflush(stdout);
    check(hy_index_set_nprobe(h, o.nprobe), "nprobe");
    check(hy_index_set_form(h, o.form), "form");
    check(hy_index_set_graph(h, o.graph), "graph");
    if (!o.train_data.empty()) insert_phase(h, o, d);
    query_phase(h, o, d);
    hy_index_destroy(h);
    std::printf("[harmony_serve] shut down\n");
    return 0;
}
