// The reference's input files, read (and written) on the host:
//  - DPD lists: a data file of fixed-size direct-access records plus a
//    ".c" sidecar of sequential unformatted records (the list's populations,
//    iops, irreps and per-irrep record offsets), as libsrint writes them
//    (clmoioso0.f:30-67 with inipckso.f / updmoiso.f, putlstso.f) and reads
//    them (getallso_d.f:31-79, getlstso.f:50-125);
//  - the "interface" node file (src/pyscf2cc/mod_interface.f90): a stream
//    file with a header (position of the node table, node count), the data
//    and a table of (name, position, size) nodes.
// The files come from gfortran (or nvfortran) builds with 8-byte default
// integers (-i8 / -fdefault-integer-8, src/make.config:110,
// src/pyscf2cc/Makefile:5): sequential records are framed by 4-byte
// little-endian length markers, direct-access records are `iprcln` bytes
// (32768, `iprcwd` = 4096 doubles, src/pyscf2cc/mod_py2cc.f90:13-16).
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "runtime.hpp"

namespace cpsd {
namespace {

constexpr int64_t REC_BYTES = 32768;  // iprcln
constexpr int64_t REC_WORDS = 4096;   // iprcwd
constexpr int NAME_LEN = 20;          // interface node names (nameLen)
constexpr int NODE_BYTES = 36;        // one node in the table (nBit): name, pos, size

std::string join(const char *dir, const std::string &name) {
    std::string d = dir ? dir : "";
    if (d.empty()) return name;
    if (d.back() != '/') d += '/';
    return d + name;
}

// the reference's 8-character file names keep trailing blanks out of the
// path (trim(filepath)//trim(filename))
std::string trim8(const char *name) {
    std::string s(name ? name : "");
    if (s.size() > 8) s.resize(8);
    while (!s.empty() && s.back() == ' ') s.pop_back();
    return s;
}

struct File {
    FILE *f = nullptr;
    File(const std::string &p, const char *mode) : f(fopen(p.c_str(), mode)) {}
    ~File() {
        if (f) fclose(f);
    }
};

// one sequential unformatted record: 4-byte length, payload, 4-byte length
int read_record(FILE *f, void *out, size_t bytes, const std::string &what) {
    uint32_t a = 0, b = 0;
    if (fread(&a, 4, 1, f) != 1) return set_error(CPSD_EARG, what + ": end of file");
    if (a != bytes)
        return set_error(CPSD_ELAYOUT, what + ": record of " + std::to_string(a) + " bytes, expected " +
                                           std::to_string(bytes) + " (8-byte integers, 4-byte markers)");
    if (fread(out, 1, bytes, f) != bytes || fread(&b, 4, 1, f) != 1 || b != a)
        return set_error(CPSD_ELAYOUT, what + ": truncated record");
    return CPSD_OK;
}
int write_record(FILE *f, const void *in, size_t bytes) {
    const uint32_t m = (uint32_t)bytes;
    if (fwrite(&m, 4, 1, f) != 1 || fwrite(in, 1, bytes, f) != bytes || fwrite(&m, 4, 1, f) != 1)
        return set_error(CPSD_EARG, "write failed");
    return CPSD_OK;
}

// node table of an interface file; pos / size as stored (1-based byte
// positions, sizes in bytes)
struct Node {
    std::string name;
    int64_t pos, size;
};
int read_nodes(FILE *f, int64_t *meta, std::vector<Node> *nodes, const std::string &path) {
    int64_t hdr[2];
    if (fseek(f, 0, SEEK_SET) != 0 || fread(hdr, 8, 2, f) != 2)
        return set_error(CPSD_EARG, path + ": no interface header");
    *meta = hdr[0];
    if (hdr[1] < 0 || hdr[1] > 1000 || hdr[0] < 17) return set_error(CPSD_ELAYOUT, path + ": bad interface header");
    nodes->clear();
    if (hdr[1] > 0 && fseek(f, (long)(hdr[0] - 1), SEEK_SET) != 0) return set_error(CPSD_ELAYOUT, path + ": bad table");
    for (int64_t i = 0; i < hdr[1]; i++) {
        unsigned char rec[NODE_BYTES];
        if (fread(rec, 1, NODE_BYTES, f) != NODE_BYTES) return set_error(CPSD_ELAYOUT, path + ": truncated table");
        Node n;
        n.name.assign((const char *)rec, NAME_LEN);
        while (!n.name.empty() && n.name.back() == ' ') n.name.pop_back();
        memcpy(&n.pos, rec + NAME_LEN, 8);
        memcpy(&n.size, rec + NAME_LEN + 8, 8);
        nodes->push_back(n);
    }
    return CPSD_OK;
}

// full_name of mod_interface.f90: blank-padded to 20 characters, lower case
std::string node_name(const char *name) {
    std::string s(name ? name : "");
    for (char &c : s)
        if (c >= 'A' && c <= 'Z') c = (char)(c + 32);
    while (!s.empty() && s.back() == ' ') s.pop_back();
    return s;
}

}  // namespace
}  // namespace cpsd

using namespace cpsd;

extern "C" {

int cpsd_dpd_list_meta_read(const char *dir, const char *name, cpsd_dpd_list_meta *m) {
    const std::string path = join(dir, trim8(name) + ".c");
    File fl(path, "rb");
    if (!fl.f) return set_error(CPSD_EARG, path + ": cannot open");
    FILE *f = fl.f;
    CPSD_TRY(read_record(f, &m->irrepx, 8, path));
    CPSD_TRY(read_record(f, m->popp, 64, path));
    CPSD_TRY(read_record(f, m->popq, 64, path));
    CPSD_TRY(read_record(f, m->popr, 64, path));
    CPSD_TRY(read_record(f, m->pops, 64, path));
    CPSD_TRY(read_record(f, m->ioppq, 64, path));
    CPSD_TRY(read_record(f, m->ioprs, 64, path));
    CPSD_TRY(read_record(f, m->irrepr, 64, path));
    CPSD_TRY(read_record(f, m->irrepi, 64, path));
    CPSD_TRY(read_record(f, m->moionuml, sizeof m->moionuml, path));
    CPSD_TRY(read_record(f, m->moionumr, sizeof m->moionumr, path));
    CPSD_TRY(read_record(f, m->rectmp, sizeof m->rectmp, path));
    return CPSD_OK;
}

// getallso of list 1 (getallso_d.f:63-79 with getlstso.f:94-125): irrep
// block R (right-pair irrep R, left irrep R x irrepx) holds
// moionuml(R) * moionumr(R) words from the first word of record
// rectmp(R) + 1; blocks follow one another in irrep order in the output
int cpsd_dpd_list_read(const char *dir, const char *name, double *host, int64_t len) {
    if (!ctx().init) return set_error(CPSD_ESTATE, "cpsd_init has not been called");
    cpsd_dpd_list_meta m;
    CPSD_TRY(cpsd_dpd_list_meta_read(dir, name, &m));
    const i64 ioppq = m.ioppq[0], ioprs = m.ioprs[0], irrepx = m.irrepr[0];
    const i64 want = idsymsoc(irrepx, m.popp, m.popq, ioppq, m.popr, m.pops, ioprs);
    if (want != len)
        return set_error(CPSD_ELAYOUT, trim8(name) + ": the list holds " + std::to_string(want) +
                                           " elements, the caller's array " + std::to_string(len));
    const std::string path = join(dir, trim8(name));
    File fl(path, "rb");
    if (!fl.f) return set_error(CPSD_EARG, path + ": cannot open");
    i64 off = 0;
    for (i64 R = 1; R <= ctx().nirrep; R++) {
        const i64 L = dp(R, irrepx);
        const i64 numl = irpdso(L, m.popp, m.popq, ioppq), numr = irpdso(R, m.popr, m.pops, ioprs);
        const i64 n = numl * numr;
        if (n == 0) continue;
        if (m.moionuml[0][R - 1] != numl || m.moionumr[0][R - 1] != numr)
            return set_error(CPSD_ELAYOUT, path + ": block sizes of irrep " + std::to_string(R) +
                                               " differ from the populations");
        const i64 rec0 = m.rectmp[0][R - 1];  // records before the block
        if (fseek(fl.f, (long)(rec0 * REC_BYTES), SEEK_SET) != 0 ||
            fread(host + off, sizeof(double), (size_t)n, fl.f) != (size_t)n)
            return set_error(CPSD_ELAYOUT, path + ": truncated data of irrep " + std::to_string(R));
        off += n;
    }
    return CPSD_OK;
}

// clmoioso0 (list 1) followed by putlstso of every distribution: the
// sidecar with rectmp(R + 1) = rectmp(R) + ceil(numl numr / iprcwd)
// (updmoiso.f:50-75) and the data records, each irrep block from the start
// of its first record, zero-padded to whole records
int cpsd_dpd_list_write(const char *dir, const char *name, int64_t irrepx, const int64_t *popp, const int64_t *popq,
                        int64_t ioppq, const int64_t *popr, const int64_t *pops, int64_t ioprs, const double *host) {
    if (!ctx().init) return set_error(CPSD_ESTATE, "cpsd_init has not been called");
    const std::string path = join(dir, trim8(name));
    cpsd_dpd_list_meta m;
    memset(&m, 0, sizeof m);
    m.irrepx = irrepx;
    memcpy(m.popp, popp, 64);
    memcpy(m.popq, popq, 64);
    memcpy(m.popr, popr, 64);
    memcpy(m.pops, pops, 64);
    m.ioppq[0] = ioppq;
    m.ioprs[0] = ioprs;
    m.irrepr[0] = irrepx;
    {
        File fl(path, "wb");
        if (!fl.f) return set_error(CPSD_EARG, path + ": cannot create");
        std::vector<double> rec((size_t)REC_WORDS);
        i64 off = 0, records = 0;
        for (i64 R = 1; R <= ctx().nirrep; R++) {
            const i64 L = dp(R, irrepx);
            const i64 numl = irpdso(L, popp, popq, ioppq), numr = irpdso(R, popr, pops, ioprs);
            const i64 n = numl * numr, nrec = (n + REC_WORDS - 1) / REC_WORDS;
            m.moionuml[0][R - 1] = numl;
            m.moionumr[0][R - 1] = numr;
            m.rectmp[0][R - 1] = records;
            for (i64 r = 0; r < nrec; r++) {
                const i64 w = std::min(REC_WORDS, n - r * REC_WORDS);
                std::fill(rec.begin(), rec.end(), 0.0);
                memcpy(rec.data(), host + off + r * REC_WORDS, sizeof(double) * (size_t)w);
                if (fwrite(rec.data(), sizeof(double), (size_t)REC_WORDS, fl.f) != (size_t)REC_WORDS)
                    return set_error(CPSD_EARG, path + ": write failed");
            }
            off += n;
            records += nrec;
        }
        // updmoiso.f:60-65: the record after the last irrep starts list 2
        m.rectmp[1][0] = records;
    }
    File fc(path + ".c", "wb");
    if (!fc.f) return set_error(CPSD_EARG, path + ".c: cannot create");
    FILE *f = fc.f;
    CPSD_TRY(write_record(f, &m.irrepx, 8));
    CPSD_TRY(write_record(f, m.popp, 64));
    CPSD_TRY(write_record(f, m.popq, 64));
    CPSD_TRY(write_record(f, m.popr, 64));
    CPSD_TRY(write_record(f, m.pops, 64));
    CPSD_TRY(write_record(f, m.ioppq, 64));
    CPSD_TRY(write_record(f, m.ioprs, 64));
    CPSD_TRY(write_record(f, m.irrepr, 64));
    CPSD_TRY(write_record(f, m.irrepi, 64));
    CPSD_TRY(write_record(f, m.moionuml, sizeof m.moionuml));
    CPSD_TRY(write_record(f, m.moionumr, sizeof m.moionumr));
    CPSD_TRY(write_record(f, m.rectmp, sizeof m.rectmp));
    return CPSD_OK;
}

int cpsd_interface_size(const char *path, const char *node, int64_t *bytes) {
    File fl(path, "rb");
    if (!fl.f) return set_error(CPSD_EARG, std::string(path) + ": cannot open");
    int64_t meta;
    std::vector<Node> nodes;
    CPSD_TRY(read_nodes(fl.f, &meta, &nodes, path));
    const std::string want = node_name(node);
    for (const Node &n : nodes)
        if (n.name == want) {
            *bytes = n.size;
            return CPSD_OK;
        }
    return set_error(CPSD_EARG, std::string(path) + ": node '" + want + "' not found");
}

// read_node_* (mod_interface.f90:518-820): the node's size must equal the
// caller's buffer
int cpsd_interface_read(const char *path, const char *node, void *out, int64_t bytes) {
    File fl(path, "rb");
    if (!fl.f) return set_error(CPSD_EARG, std::string(path) + ": cannot open");
    int64_t meta;
    std::vector<Node> nodes;
    CPSD_TRY(read_nodes(fl.f, &meta, &nodes, path));
    const std::string want = node_name(node);
    for (const Node &n : nodes)
        if (n.name == want) {
            if (n.size != bytes)
                return set_error(CPSD_ELAYOUT, "node '" + want + "' holds " + std::to_string(n.size) +
                                                   " bytes, the caller asked for " + std::to_string(bytes));
            if (fseek(fl.f, (long)(n.pos - 1), SEEK_SET) != 0 || fread(out, 1, (size_t)bytes, fl.f) != (size_t)bytes)
                return set_error(CPSD_ELAYOUT, "node '" + want + "': truncated data");
            return CPSD_OK;
        }
    return set_error(CPSD_EARG, std::string(path) + ": node '" + want + "' not found");
}

// add_node_* (mod_interface.f90:80-130, 227-500): a new node's data goes at
// the table position, the table moves behind it; a node written again keeps
// its place when the data is not longer, else moves behind the data
int cpsd_interface_write(const char *path, const char *node, const void *data, int64_t bytes) {
    const std::string want = node_name(node);
    if (want.empty() || want.size() > NAME_LEN) return set_error(CPSD_EARG, "node names have 1..20 characters");
    int64_t meta = 17;
    std::vector<Node> nodes;
    {
        File fr(path, "rb");
        if (fr.f) CPSD_TRY(read_nodes(fr.f, &meta, &nodes, path));
    }
    File fl(path, nodes.empty() && meta == 17 ? "w+b" : "r+b");
    if (!fl.f) return set_error(CPSD_EARG, std::string(path) + ": cannot open for writing");
    Node *hit = nullptr;
    for (Node &n : nodes)
        if (n.name == want) hit = &n;
    if (!hit) {
        if (nodes.size() >= 1000) return set_error(CPSD_EARG, "interface files hold at most 1000 nodes");
        nodes.push_back({want, meta, bytes});
        hit = &nodes.back();
        meta += bytes;
    } else if (hit->size < bytes) {
        hit->pos = meta;
        hit->size = bytes;
        meta += bytes;
    } else {
        hit->size = bytes;
    }
    if (fseek(fl.f, (long)(hit->pos - 1), SEEK_SET) != 0 || fwrite(data, 1, (size_t)bytes, fl.f) != (size_t)bytes)
        return set_error(CPSD_EARG, "node '" + want + "': write failed");
    const int64_t hdr[2] = {meta, (int64_t)nodes.size()};
    if (fseek(fl.f, 0, SEEK_SET) != 0 || fwrite(hdr, 8, 2, fl.f) != 2)
        return set_error(CPSD_EARG, std::string(path) + ": header write failed");
    if (fseek(fl.f, (long)(meta - 1), SEEK_SET) != 0) return set_error(CPSD_EARG, "table seek failed");
    for (const Node &n : nodes) {
        unsigned char rec[NODE_BYTES];
        memset(rec, ' ', NAME_LEN);
        memcpy(rec, n.name.data(), n.name.size());
        memcpy(rec + NAME_LEN, &n.pos, 8);
        memcpy(rec + NAME_LEN + 8, &n.size, 8);
        if (fwrite(rec, 1, NODE_BYTES, fl.f) != NODE_BYTES) return set_error(CPSD_EARG, "table write failed");
    }
    return CPSD_OK;
}

// readmodule (src/lib_cc/readmodule.f90:17-40): symry, dirprd, nirrep, and
// pop / vrt as (8, 2) arrays (alpha, beta)
int cpsd_load_system(const char *interface_path, cpsd_system *s) {
    memset(s, 0, sizeof *s);
    int64_t pop[16], vrt[16];
    CPSD_TRY(cpsd_interface_read(interface_path, "symry", &s->symry, 8));
    CPSD_TRY(cpsd_interface_read(interface_path, "dirprd", s->dirprd, 64 * 8));
    CPSD_TRY(cpsd_interface_read(interface_path, "nirrep", &s->nirrep, 8));
    CPSD_TRY(cpsd_interface_read(interface_path, "pop", pop, sizeof pop));
    CPSD_TRY(cpsd_interface_read(interface_path, "vrt", vrt, sizeof vrt));
    for (int h = 0; h < 8; h++) {
        s->popa[h] = pop[h];
        s->popb[h] = pop[8 + h];
        s->vrta[h] = vrt[h];
        s->vrtb[h] = vrt[8 + h];
    }
    if (s->nirrep < 1 || s->nirrep > 8) return set_error(CPSD_ELAYOUT, "interface: nirrep out of range");
    return CPSD_OK;
}

// the programs' input (loadSCF.f90:13-48 of EE-CIS.SF / CPSd.SF /
// EE-CPSd.SF): the spin-free orbital energies ('orb_energy_no_spin', nvir +
// nocc values) and the six integral lists 'ijkl_ns_' ... 'abcd_ns_'
// (src/EE-CPSd.SF/mod_variable.f90:37-47) in the layouts of allocate_mem.f90
// (iop 0 on antisymmetric pairs); dir NULL: the interface's 'tmpdir' node,
// else the current directory (get_f_path.f90)
int cpsd_load_inputs(const char *dir, const char *interface_path, const cpsd_system *s, double *ijkl, double *ijka,
                     double *abij, double *iabj, double *abci, double *abcd, double *eorb) {
    CPSD_TRY(cpsd_init(s->nirrep, s->dirprd));
    i64 popo[8] = {}, popv[8] = {};
    for (i64 r = 1; r <= s->nirrep; r++) {
        const i64 rb = dp(r, s->symry);
        popo[r - 1] = s->popa[r - 1] + s->popb[rb - 1];
        popv[r - 1] = s->vrta[r - 1] + s->vrtb[rb - 1];
    }
    std::string d = dir ? dir : "";
    if (!dir) {
        int64_t n = 0;
        if (cpsd_interface_size(interface_path, "tmpdir", &n) == CPSD_OK && n > 0 && n < 4096) {
            std::vector<char> buf((size_t)n);
            CPSD_TRY(cpsd_interface_read(interface_path, "tmpdir", buf.data(), n));
            d.assign(buf.data(), buf.size());
            while (!d.empty() && (d.back() == ' ' || d.back() == 0)) d.pop_back();
        }
    }
    struct L {
        const char *name;
        double *out;
        const i64 *p[4];
        i64 iop[2];
    } lists[6] = {{"ijkl_ns_", ijkl, {popo, popo, popo, popo}, {0, 0}},
                  {"ijka_ns_", ijka, {popo, popo, popo, popv}, {0, 1}},
                  {"abij_ns_", abij, {popv, popv, popo, popo}, {0, 0}},
                  {"iabj_ns_", iabj, {popv, popo, popv, popo}, {1, 1}},
                  {"abci_ns_", abci, {popv, popv, popv, popo}, {0, 1}},
                  {"abcd_ns_", abcd, {popv, popv, popv, popv}, {0, 0}}};
    for (const L &l : lists) {
        if (!l.out) continue;
        cpsd_dpd_list_meta m;
        CPSD_TRY(cpsd_dpd_list_meta_read(d.c_str(), l.name, &m));
        const i64 *mp[4] = {m.popp, m.popq, m.popr, m.pops};
        for (int k = 0; k < 4; k++)
            if (memcmp(mp[k], l.p[k], 8 * sizeof(i64)) != 0)
                return set_error(CPSD_ELAYOUT, std::string(l.name) + ": populations differ from the system's");
        if (m.ioppq[0] != l.iop[0] || m.ioprs[0] != l.iop[1] || m.irrepr[0] != 1)
            return set_error(CPSD_ELAYOUT, std::string(l.name) + ": iops or irrep differ from the programs' layout");
        const i64 len = idsymsoc(1, l.p[0], l.p[1], l.iop[0], l.p[2], l.p[3], l.iop[1]);
        CPSD_TRY(cpsd_dpd_list_read(d.c_str(), l.name, l.out, len));
    }
    if (eorb) {
        i64 n = 0;
        for (int r = 0; r < 8; r++) n += popo[r] + popv[r];
        CPSD_TRY(cpsd_interface_read(interface_path, "orb_energy_no_spin", eorb, 8 * n));
    }
    return CPSD_OK;
}

}  // extern "C"
