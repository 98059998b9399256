// gtb_reader.cpp -- host reader and packer: PDB structure files (plain or
// gzip-compressed) into one block of the reference's SoA fields, the input of
// gtb_process_block / gtb_block_upload.  Host code; files are parsed in
// parallel on host threads and packed in file order.
//
// The record loop follows FlexDataRead::ReadDataPDB
// (src/libgenp/gdats/FlexDataRead.cpp:285-560) step for step, including its
// byte-offset line handling (myfiler.h:56-64: a skip of `by` bytes moves
// past the end of the line it lands in, so a record shorter than the skip
// also skips the next line), because the structures a file yields depend on
// it: the --ter / --split rules, the alternate-location filter (' ' or 'A'),
// ATOM (and, with --hetatm, HETATM) records of the --aatom / --natom atom,
// the --mol molecule-type vote, the --dev-min-length / --dev-max-length
// limits (PMBatchStrData.h:368-415, 440-460) and the description format
// (PMBatchStrData.h:525-545).  Residue codes: ResName2Code
// (src/libutil/alpha.cpp:65-75, 115-143).  Field values as AddOneResidue
// writes them (PM2DVectorFields.h:40-41, 96-115): per residue
// (insertion code << 16 | chain id << 8 | chain order), negated for protein
// residues; per structure the length, the offset of its first residue and
// the molecule-type vote (pps2DType outside clustering runs).
// PDBx/mmCIF files follow FlexDataRead::ReadDataCIF (FlexDataRead.cpp:553-
// 930): the _atom_site loop's columns, tokens of a record's first 128
// characters, the model / chain changes as structure ends.  The format comes
// from the file name as InputFilelist::GetFileTypeFromFilename decides it
// (InputFilelist.h:147-174: .cif / .cif.gz are PDBx/mmCIF, anything else
// PDB, unless the --infmt option says which); files under 10 bytes are
// skipped (InputFilelist.h AddFile).  Tar archives are read entry by entry
// as InputFilelist::AddFilesFromTAR lists them (InputFilelist.cpp:95-200:
// regular files of 10 bytes to 128 MB, a bad header checksum ends the list,
// each entry's format from its name, gzip entries inflated), the
// description being "<archive>:<entry>" (FlexDataRead.h:219-222).

#include <zlib.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "gtb200.h"

namespace {

enum { TER_EOF = 0, TER_END = 1, TER_END_CHAIN = 2, TER_TER_END_CHAIN = 3 };
enum { SPLIT_NONE = 0, SPLIT_MODEL = 1, SPLIT_CHAIN = 2 };

// one-letter code of a residue name (3 characters at p)
char res_code(const char* p) {
    static const char* const names[] = {
        "ALA", "DAL", "ASX", "CYS", "DCY", "ASP", "DAS", "GLU", "DGL", "PHE", "DPN", "GLY",
        "HIS", "DHI", "ILE", "DIL", "LYS", "DLY", "LEU", "DLE", "MET", "MED", "MSE", "ASN",
        "DSG", "PYL", "PRO", "DPR", "GLN", "DGN", "ARG", "DAR", "SER", "DSN", "THR", "DTH",
        "SEC", "VAL", "DVA", "TRP", "DTR", "TYR", "DTY", "GLX"};
    static const char codes[] = "AABCCDDEEFFGHHIIKKLLMMMNNOPPQQRRSSTTUVVWWYYZ";
    // the names are three capital letters: a 26^3 table, built once
    static const std::vector<char> table = []() {
        std::vector<char> t(26 * 26 * 26, 0);
        for (size_t k = 0; k < sizeof(names) / sizeof(names[0]); k++)
            t[(size_t)((names[k][0] - 'A') * 676 + (names[k][1] - 'A') * 26 + (names[k][2] - 'A'))] = codes[k];
        return t;
    }();
    if (p[0] >= 'A' && p[0] <= 'Z' && p[1] >= 'A' && p[1] <= 'Z' && p[2] >= 'A' && p[2] <= 'Z') {
        const char c = table[(size_t)((p[0] - 'A') * 676 + (p[1] - 'A') * 26 + (p[2] - 'A'))];
        if (c) return c;
    }
    // names of one or two characters (nucleotides): the letter itself
    if (p[0] == ' ') {
        if (p[1] == ' ') return p[2] == ' ' ? 'X' : p[2];
        return p[2] == ' ' ? p[1] : 'X';
    }
    return p[1] == ' ' ? p[0] : 'X';
}

struct Structure {
    std::string desc;
    std::vector<float> x, y, z;
    std::vector<int> insch, resnum;
    std::vector<char> rsd;
    int moltype = 0;
    void clear() {
        x.clear(); y.clear(); z.clear(); insch.clear(); resnum.clear(); rsd.clear();
    }
};

struct FileResult {
    std::vector<Structure> strs;
    std::string err;          // empty: read
};

bool read_raw(const char* path, std::string& buf) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return false;
    buf.clear();
    char tmp[1 << 16];
    size_t n;
    while ((n = std::fread(tmp, 1, sizeof(tmp), f)) > 0) buf.append(tmp, n);
    std::fclose(f);
    return true;
}

bool read_all(const char* path, std::string& buf, std::string& err) {
    gzFile f = gzopen(path, "rb");     // reads plain files as they are
    if (!f) { err = std::string("cannot open ") + path; return false; }
    buf.clear();
    char tmp[1 << 16];
    for (;;) {
        int n = gzread(f, tmp, sizeof(tmp));
        if (n < 0) { int e = 0; err = std::string(path) + ": " + gzerror(f, &e); gzclose(f); return false; }
        if (n == 0) break;
        buf.append(tmp, (size_t)n);
    }
    gzclose(f);
    return true;
}

// the leading integer / number of a fixed-width field, as std::stoi / std::stof
// read it (leading blanks skipped, trailing characters ignored); false: none
bool field_int(const char* p, int w, int& v) {
    // the common form: [blanks][sign] up to 9 digits
    int k = 0;
    while (k < w && (p[k] == ' ' || p[k] == '\t' || p[k] == '\n' || p[k] == '\r' ||
                     p[k] == '\v' || p[k] == '\f')) k++;
    bool neg = false;
    if (k < w && (p[k] == '-' || p[k] == '+')) { neg = p[k] == '-'; k++; }
    int nd = 0;
    long r0 = 0;
    for (; k < w && p[k] >= '0' && p[k] <= '9' && nd < 10; k++, nd++) r0 = r0 * 10 + (p[k] - '0');
    if (nd > 0 && nd <= 9 && !(k < w && p[k] >= '0' && p[k] <= '9')) {
        v = (int)(neg ? -r0 : r0);
        return true;
    }
    char s[32];
    const int n = w < 31 ? w : 31;
    std::memcpy(s, p, (size_t)n);
    s[n] = 0;
    char* e = nullptr;
    long r = std::strtol(s, &e, 10);
    if (e == s) return false;
    v = (int)r;
    return true;
}
bool field_float(const char* p, int w, float& v) {
    // the common form, [blanks][sign]digits[.digits] with at most 9 digits and
    // 6 decimals: m / 10^d in double is the correctly rounded quotient (both
    // exact in double; Clinger's fast path), and its rounding to float is the
    // correctly rounded float of the decimal (a decimal of at most 6 places
    // lies at least ulp/(2*10^6) from any float midpoint it is not equal to,
    // far beyond the double's error), so this equals strtof
    int k = 0;
    while (k < w && (p[k] == ' ' || p[k] == '\t')) k++;
    bool neg = false;
    if (k < w && (p[k] == '-' || p[k] == '+')) { neg = p[k] == '-'; k++; }
    long long m = 0;
    int nd = 0, dec = -1, j = k;
    for (; j < w; j++) {
        const char c = p[j];
        if (c >= '0' && c <= '9') { m = m * 10 + (c - '0'); nd++; if (dec >= 0) dec++; }
        else if (c == '.' && dec < 0) dec = 0;
        else break;
    }
    const bool end = j == w || p[j] == ' ' || p[j] == '\t' || p[j] == '\n' || p[j] == '\r';
    if (nd > 0 && nd <= 9 && dec <= 6 && end) {
        static const double p10[7] = {1e0, 1e1, 1e2, 1e3, 1e4, 1e5, 1e6};
        const double q = (double)m / p10[dec < 0 ? 0 : dec];
        v = (float)(neg ? -q : q);
        return true;
    }
    char s[32];
    const int n = w < 31 ? w : 31;
    std::memcpy(s, p, (size_t)n);
    s[n] = 0;
    char* e = nullptr;
    float r = std::strtof(s, &e);
    if (e == s) return false;
    v = r;
    return true;
}

void parse_pdb(const std::string& path, const std::string& data, const gtb_reader_options& o,
               FileResult& out) {
    const size_t terlnwidth = 26, sfflnwidth = 54, sffmodlnwidth = 12;
    const int ter = o.ter, split = o.split;
    const bool usechid = !(ter == TER_EOF && (split == SPLIT_NONE || split == SPLIT_MODEL));
    const bool usemodn = !(ter == TER_EOF && split == SPLIT_NONE);
    const char* data0 = data.data();
    const size_t datlen = data.size();
    size_t cur = 0;
    auto incposnl = [&](size_t by) {
        cur += by;
        size_t p = cur;
        while (p < datlen && data0[p] != '\n' && data0[p] != '\r') p++;
        while (p < datlen && (data0[p] == '\n' || data0[p] == '\r')) p++;
        cur = p;
    };
    int moltype = 0;
    char chord = 0, prevchid = 0, prevchidx = 0;
    std::string model, modelprev;
    Structure s;
    const size_t guess = data.size() / 81 + 1;  // a residue per 80-column record, at most
    s.x.reserve(guess); s.y.reserve(guess); s.z.reserve(guess);
    s.insch.reserve(guess); s.resnum.reserve(guess); s.rsd.reserve(guess);
    bool stop = false;          // file closed (the reader's Eof)
    // FinalizeCrntStructure: 0 written, 1 empty, 2 short, 3 (never: too long
    // structures are dropped while being added)
    auto finalize = [&](char chain, const std::string& mdl) -> int {
        const int n = (int)s.x.size();
        int code = 0;
        if (n < 1) code = 1;
        else if (n < o.minlen) code = 2;
        else {
            std::string d = path;
            if (usechid && chain) d += std::string(" Chn:") + chain;
            if (usemodn && !mdl.empty()) d += " (M:" + mdl + ")";
            s.desc = d;
            s.moltype = moltype;
            out.strs.push_back(s);
        }
        s.clear();
        return code;
    };
    // a record's bytes past the end of the data read as zeros
    auto at = [&](size_t k) -> char { return k < datlen ? data0[k] : '\0'; };
    auto cmp = [&](size_t k, const char* lit) {
        for (size_t i = 0; lit[i]; i++) if (at(k + i) != lit[i]) return false;
        return true;
    };
    while (!stop && cur < datlen) {
        const size_t p = cur;
        const size_t datwidth = datlen - p;
        if (datwidth < 3) { incposnl(0); continue; }
        if (!s.x.empty()) {
            if ((ter >= TER_END && cmp(p, "END")) || (ter >= TER_TER_END_CHAIN && cmp(p, "TER"))) {
                stop = true;
                break;
            }
        }
        if (split > SPLIT_NONE && cmp(p, "END")) {
            prevchid = 0;
            incposnl(3);
            continue;
        }
        if (cmp(p, "MODEL ") && datwidth > sffmodlnwidth) {
            std::string m;
            for (size_t i = 10; i < 14 && at(p + i) != '\n' && at(p + i) != '\r'; i++)
                if (at(p + i) != ' ' && at(p + i) != '\t') m += at(p + i);
            model = m;                  // at most the 4 characters of columns 11-14
            incposnl(sffmodlnwidth);
            continue;
        }
        if (datwidth < sfflnwidth || (at(p + 16) != ' ' && at(p + 16) != 'A')) {
            incposnl(0);
            continue;
        }
        if (!cmp(p, "ATOM  ") && (!o.hetatm || !cmp(p, "HETATM"))) {
            incposnl(cmp(p, "TER") ? terlnwidth : sfflnwidth);
            continue;
        }
        const bool isa = std::memcmp(data0 + p + 12, o.aatom, 4) == 0;
        const bool isn = std::memcmp(data0 + p + 12, o.natom, 4) == 0;
        if (!isa && !isn) {
            incposnl(sfflnwidth);
            continue;
        }
        const char chid = data0[p + 21], insc = data0[p + 26];
        const char resd = res_code(data0 + p + 17);
        int resnum = 0;
        float c[3];
        if (!field_int(data0 + p + 22, 4, resnum) || !field_float(data0 + p + 30, 8, c[0]) ||
            !field_float(data0 + p + 38, 8, c[1]) || !field_float(data0 + p + 46, 8, c[2])) {
            out.err = path + ": failed to read residue data";
            return;
        }
        if (prevchid != chid) {
            const bool cond1 = ter >= TER_END_CHAIN;
            const bool cond2 = split == SPLIT_CHAIN || (prevchid == 0 && split == SPLIT_MODEL);
            if (!s.x.empty() && (cond1 || cond2)) {
                chord = 0;
                const int code = finalize(prevchidx, modelprev);
                if (code == 1) return;             // empty: the file is done
                if (cond1) return;
                moltype = 0;
            }
            modelprev = model;
            prevchid = prevchidx = chid;
            chord++;
        }
        int restype;
        if (o.mol == 0) restype = -1;
        else if (o.mol == 1) restype = 1;
        else restype = (data0[p + 17] == ' ' && (data0[p + 18] == ' ' || data0[p + 18] == 'D')) ? 1 : -1;
        moltype += restype;
        // the length limits compare the residues stored before this one
        // (PMBatchStrData.h:377-385)
        const int nprev = (int)s.x.size();
        if ((o.maxlen > 0 && o.maxlen < nprev) || 65535 < nprev) {
            s.clear();                             // too long: dropped, the file is done
            return;
        }
        int v = (int)((((unsigned)(unsigned char)insc & 0xffu) << 16) |
                      (((unsigned)(unsigned char)chid & 0xffu) << 8) | ((unsigned)(unsigned char)chord & 0xffu));
        v = std::abs(v);
        if (restype <= 0) v = -v;
        s.x.push_back(c[0]); s.y.push_back(c[1]); s.z.push_back(c[2]);
        s.insch.push_back(v);
        s.resnum.push_back(resnum);
        s.rsd.push_back(resd);
        incposnl(sfflnwidth);
    }
    finalize(prevchidx, modelprev);
}

// the _atom_site columns the reader uses (FlexDataRead.h's field indices)
enum CifField { CF_GROUP, CF_ATOM, CF_ALT, CF_COMP, CF_LASYM, CF_LSEQ, CF_INS, CF_X, CF_Y, CF_Z,
                CF_ASEQ, CF_AASYM, CF_MODEL, CF_SET, CF_N };

void parse_cif(const std::string& path, const std::string& data, const gtb_reader_options& o,
               FileResult& out) {
    const size_t maxlnwidth = 128, sfflnwidth = 54;
    const int ter = o.ter, split = o.split;
    const bool usechid = !(ter == TER_EOF && (split == SPLIT_NONE || split == SPLIT_MODEL));
    const bool usemodn = !(ter == TER_EOF && split == SPLIT_NONE);
    // the trimmed atom names
    auto trim = [](const char* a) {
        std::string t(a, strnlen(a, 4));
        size_t b = t.find_first_not_of(' '), e = t.find_last_not_of(' ');
        return b == std::string::npos ? std::string() : t.substr(b, e - b + 1);
    };
    const std::string satom = trim(o.aatom), natom = trim(o.natom);
    const char* d0 = data.data();
    const size_t datlen = data.size();
    auto at = [&](size_t k) -> char { return k < datlen ? d0[k] : '\0'; };
    size_t cur = 0;
    auto incposnl = [&](size_t by) {
        cur += by;
        size_t p = cur;
        while (p < datlen && d0[p] != '\n' && d0[p] != '\r') p++;
        while (p < datlen && (d0[p] == '\n' || d0[p] == '\r')) p++;
        cur = p;
    };
    int fld[CF_N];
    auto reset = [&]() { for (int& f : fld) f = -1; };
    reset();
    auto pre = [&](size_t p, size_t dw, const char* lit) {
        const size_t n = std::strlen(lit);
        if (dw < n) return false;
        for (size_t i = 0; i < n; i++) if (at(p + i) != lit[i]) return false;
        return true;
    };
    auto isspc = [](char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\v' || c == '\f'; };
    auto set_field = [&](size_t p, size_t dw, int ndx) {
        if (pre(p, dw, "group_PDB")) fld[CF_GROUP] = ndx;
        else if (pre(p, dw, "label_atom_id")) fld[CF_ATOM] = ndx;
        else if (pre(p, dw, "label_alt_id")) fld[CF_ALT] = ndx;
        else if (pre(p, dw, "label_comp_id")) fld[CF_COMP] = ndx;
        else if (pre(p, dw, "label_asym_id")) fld[CF_LASYM] = ndx;
        else if (pre(p, dw, "label_seq_id")) fld[CF_LSEQ] = ndx;
        else if (pre(p, dw, "pdbx_PDB_ins_code")) fld[CF_INS] = ndx;
        else if (pre(p, dw, "Cartn_x") && isspc(at(p + 7))) fld[CF_X] = ndx;
        else if (pre(p, dw, "Cartn_y") && isspc(at(p + 7))) fld[CF_Y] = ndx;
        else if (pre(p, dw, "Cartn_z") && isspc(at(p + 7))) fld[CF_Z] = ndx;
        else if (pre(p, dw, "auth_seq_id")) fld[CF_ASEQ] = ndx;
        else if (pre(p, dw, "auth_asym_id")) fld[CF_AASYM] = ndx;
        else if (pre(p, dw, "pdbx_PDB_model_num")) fld[CF_MODEL] = ndx;
        if (0 <= fld[CF_GROUP] && 0 <= fld[CF_ATOM] && 0 <= fld[CF_COMP] &&
            (0 <= fld[CF_AASYM] || 0 <= fld[CF_LASYM]) && (0 <= fld[CF_ASEQ] || 0 <= fld[CF_LSEQ]) &&
            0 <= fld[CF_X] && 0 <= fld[CF_Y] && 0 <= fld[CF_Z])
            fld[CF_SET] = 1;
    };
    // the atom name token matches `atom` (an opening quote skipped)
    auto check_atom = [&](size_t pt, const std::string& atom) {
        if (at(pt) == '"') pt++;
        for (size_t i = 0; i < atom.size(); i++) if (atom[i] != at(pt++)) return false;
        const char c = at(pt);
        return c == '"' || c == ' ' || c == '\t' || c == '\n' || c == '\r';
    };
    std::string modelprev(4, '\0'), chainprev(5, '\0'), model, chain;
    int loop = -1, moltype = 0;
    char chord = 0;
    Structure s;
    auto finalize = [&](const std::string& ch, const std::string& mdl) -> int {
        const int n = (int)s.x.size();
        int code = 0;
        if (n < 1) code = 1;
        else if (n < o.minlen) code = 2;
        else {
            std::string d = path;
            if (usechid && ch.size() && ch[0]) d += " Chn:" + ch;
            if (usemodn && mdl.size() && mdl[0]) d += " (M:" + mdl + ")";
            s.desc = d;
            s.moltype = moltype;
            out.strs.push_back(s);
        }
        s.clear();
        return code;
    };
    std::vector<size_t> tk, te;
    tk.reserve(maxlnwidth); te.reserve(maxlnwidth);
    while (cur < datlen) {
        const size_t pbeg = cur;
        size_t p = pbeg;
        const size_t datwidth = datlen - p;
        if (datwidth < 5 || d0[p] == '#') { reset(); incposnl(0); continue; }
        if (pre(p, datwidth, "loop_")) { reset(); loop = 0; incposnl(5); continue; }
        if (0 <= loop && (datwidth < 11 || !pre(p, datwidth, "_atom_site."))) loop = -1;
        if (0 <= loop) { set_field(p + 11, datwidth - 11, loop++); incposnl(11); continue; }
        if (fld[CF_SET] <= 0) { incposnl(0); continue; }
        // tokens of the record's first maxlnwidth characters
        tk.clear(); te.clear();
        for (const size_t pmax = p + maxlnwidth; p < datlen && p < pmax && d0[p] != '\n' && d0[p] != '\r';) {
            for (; p < datlen && p < pmax && (d0[p] == ' ' || d0[p] == '\t'); p++) {}
            tk.push_back(p);
            for (; p < datlen && p < pmax && d0[p] != ' ' && d0[p] != '\t' && d0[p] != '\n' && d0[p] != '\r'; p++) {}
            te.push_back(p);
        }
        const int nt = (int)tk.size();
        auto skip = [&]() { incposnl(p - pbeg); };
        if (nt < 1 || datwidth < sfflnwidth) { skip(); continue; }
        auto tok = [&](int f) { return tk[(size_t)fld[f]]; };
        auto toklen = [&](int f) { return te[(size_t)fld[f]] - tk[(size_t)fld[f]]; };
        if (nt <= fld[CF_GROUP] || (!pre(tok(CF_GROUP), datlen - tok(CF_GROUP), "ATOM") &&
                                    (!o.hetatm || !pre(tok(CF_GROUP), datlen - tok(CF_GROUP), "HETATM")))) {
            skip(); continue;
        }
        if (0 <= fld[CF_ALT] && (nt <= fld[CF_ALT] || (at(tok(CF_ALT)) != '.' && at(tok(CF_ALT)) != 'A'))) {
            skip(); continue;
        }
        if (nt <= fld[CF_ATOM] || (!check_atom(tok(CF_ATOM), satom) && !check_atom(tok(CF_ATOM), natom))) {
            skip(); continue;
        }
        if (nt <= fld[CF_X] || nt <= fld[CF_Y] || nt <= fld[CF_Z] || nt <= fld[CF_LSEQ] ||
            nt <= fld[CF_LASYM] || nt <= fld[CF_COMP]) {
            skip(); continue;
        }
        int fa = CF_LASYM;
        if (0 <= fld[CF_AASYM] && fld[CF_AASYM] < nt) fa = CF_AASYM;
        int fs = CF_LSEQ;
        if (0 <= fld[CF_ASEQ] && fld[CF_ASEQ] < nt) fs = CF_ASEQ;
        // a record without the chain or number column it would read (the
        // table has only the other form, past this record's tokens): skipped
        if (fld[fa] < 0 || fld[fs] < 0) { skip(); continue; }
        if (toklen(fa) < 1) { out.err = path + ": invalid PDBx/mmCIF file format"; return; }
        chain.assign(d0 + tok(fa), toklen(fa));
        char chid = chain[0];
        if (chid == '.') chid = ' ';
        char insc = ' ';
        if (0 <= fld[CF_INS] && fld[CF_INS] < nt) insc = at(tok(CF_INS));
        if (insc == '?') insc = ' ';
        char nm[3] = {at(tok(CF_COMP)), at(tok(CF_COMP) + 1), at(tok(CF_COMP) + 2)};
        const char resd = res_code(nm);
        int resnum = 0;
        float c[3];
        if (!field_int(d0 + tok(fs), (int)toklen(fs), resnum) ||
            !field_float(d0 + tok(CF_X), (int)toklen(CF_X), c[0]) ||
            !field_float(d0 + tok(CF_Y), (int)toklen(CF_Y), c[1]) ||
            !field_float(d0 + tok(CF_Z), (int)toklen(CF_Z), c[2])) {
            out.err = path + ": failed to read residue data";
            return;
        }
        bool seteof = false, fin = false;
        if (0 <= fld[CF_MODEL] && fld[CF_MODEL] < nt) {
            model.assign(d0 + tok(CF_MODEL), toklen(CF_MODEL));
            if (model != modelprev) {
                if (ter >= TER_END) { fin = true; seteof = true; }
                if (split > SPLIT_NONE) fin = true;
            }
        }
        if (chain != chainprev) {
            if (ter >= TER_END_CHAIN) { fin = true; seteof = true; }
            if (split >= SPLIT_CHAIN) fin = true;
            chord++;
        }
        if (fin && !s.x.empty()) {
            chord = 1;
            const int code = finalize(chainprev, modelprev);
            if (code == 1) return;
            if (seteof) return;
            moltype = 0;
        }
        modelprev = model;
        chainprev = chain;
        int restype;
        if (o.mol == 0) restype = -1;
        else if (o.mol == 1) restype = 1;
        else restype = (toklen(CF_COMP) < 2 || at(tok(CF_COMP)) == 'D') ? 1 : -1;
        moltype += restype;
        const int nprev = (int)s.x.size();
        if ((o.maxlen > 0 && o.maxlen < nprev) || 65535 < nprev) { s.clear(); return; }
        int v = (int)((((unsigned)(unsigned char)insc & 0xffu) << 16) |
                      (((unsigned)(unsigned char)chid & 0xffu) << 8) | ((unsigned)(unsigned char)chord & 0xffu));
        v = std::abs(v);
        if (restype <= 0) v = -v;
        s.x.push_back(c[0]); s.y.push_back(c[1]); s.z.push_back(c[2]);
        s.insch.push_back(v);
        s.resnum.push_back(resnum);
        s.rsd.push_back(resd);
        skip();
    }
    finalize(chainprev, modelprev);
}

// gzip data in memory -> out
bool gunzip(const std::string& in, std::string& out) {
    z_stream zs;
    std::memset(&zs, 0, sizeof(zs));
    if (inflateInit2(&zs, 16 + MAX_WBITS) != Z_OK) return false;
    zs.next_in = (Bytef*)in.data();
    zs.avail_in = (uInt)in.size();
    out.clear();
    char tmp[1 << 16];
    int rc = Z_OK;
    while (rc == Z_OK) {
        zs.next_out = (Bytef*)tmp;
        zs.avail_out = sizeof(tmp);
        rc = inflate(&zs, Z_NO_FLUSH);
        if (rc != Z_OK && rc != Z_STREAM_END) { inflateEnd(&zs); return false; }
        out.append(tmp, sizeof(tmp) - zs.avail_out);
        if (rc == Z_OK && zs.avail_in == 0 && zs.avail_out != 0) break;   // truncated input
    }
    inflateEnd(&zs);
    return true;
}

struct TarEntry { std::string name; size_t pos, size; };

// the regular-file entries of a tar archive (as AddFilesFromTAR lists them)
bool tar_entries(const std::string& tar, std::vector<TarEntry>& ents) {
    const size_t HS = 512;
    auto oct = [&](size_t at, int w) {
        size_t r = 0;
        const char* h = tar.data() + at;
        for (; !('0' <= *h && *h <= '7') && 0 < w; h++, w--) {}
        for (; ('0' <= *h && *h <= '7') && 0 < w; h++, w--) r = 8 * r + (size_t)(*h - '0');
        return r;
    };
    size_t pos = 0;
    for (;;) {
        if (pos + HS > tar.size()) return pos == tar.size();    // ill-formed unless at the end
        const unsigned char* h = (const unsigned char*)tar.data() + pos;
        int sum = 0, sumfld = 0;
        for (size_t n = 0; n < HS; n++) sum += h[n];
        for (size_t n = 148; n < 156; n++) sumfld += h[n];
        if (sum == 0) return true;                              // the end marker
        const int chk = (int)oct(pos + 148, 8);
        if (sum - sumfld + 8 * 32 != chk) return true;          // corrupted: the list ends
        const int type = (int)h[156];
        const size_t size = oct(pos + 124, 12);
        const size_t start = pos + HS;
        pos = start + (size + 511) / 512 * 512;
        if (type != '0' && type != 0) continue;
        if (size < 10 || size > ((size_t)128 << 20)) continue;
        if (start + size > tar.size()) return false;
        std::string name((const char*)h, strnlen((const char*)h, 100));
        ents.push_back({name, start, size});
    }
}

bool ends_with(const std::string& a, const char* b) {
    const size_t n = std::strlen(b);
    return n < a.size() && a.compare(a.size() - n, n, b) == 0;
}

// 0 PDB, 1 PDBx/mmCIF, 2 tar (refused)
int file_format(const std::string& name, int infmt) {
    if (ends_with(name, ".gz")) {
        if (infmt == 1) return 0;
        if (infmt == 2) return 1;
        if (ends_with(name, ".pdb.gz") || ends_with(name, ".ent.gz")) return 0;
        if (ends_with(name, ".cif.gz")) return 1;
        return 0;
    }
    if (ends_with(name, ".tar")) return 2;
    if (infmt == 1) return 0;
    if (infmt == 2) return 1;
    if (ends_with(name, ".cif")) return 1;
    return 0;
}

}  // namespace

struct gtb_structs {
    std::vector<Structure> strs;
    std::vector<int> len, type, insch, resnum;
    std::vector<unsigned> dist;
    std::vector<float> x, y, z;
    std::vector<char> rsd, ss;
    std::string err;
};

extern "C" void gtb_reader_default_options(gtb_reader_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->ter = TER_TER_END_CHAIN;
    o->split = SPLIT_NONE;
    o->hetatm = 0;
    o->mol = 2;
    std::memcpy(o->aatom, " CA ", 5);
    std::memcpy(o->natom, " C3'", 5);
    o->minlen = 20;
    o->maxlen = 65535;
    o->infmt = 0;
}

extern "C" gtb_status gtb_read_pdb(const char* const* paths, int npaths,
                                   const gtb_reader_options* opts, int nthreads,
                                   gtb_structs** out, char* err, size_t errlen) {
    auto fail = [&](gtb_status st, const std::string& m) {
        if (err && errlen) std::snprintf(err, errlen, "%s", m.c_str());
        return st;
    };
    if (!out || npaths < 0 || (npaths > 0 && !paths)) return fail(GTB_ERR_ARG, "bad arguments");
    *out = nullptr;
    gtb_reader_options o;
    if (opts) o = *opts;
    else gtb_reader_default_options(&o);
    if (o.ter < 0 || o.ter > 3 || o.split < 0 || o.split > 2 || o.mol < 0 || o.mol > 2 ||
        o.minlen < 1 || o.maxlen < 0 || o.maxlen > 65535 || o.infmt < 0 || o.infmt > 2)
        return fail(GTB_ERR_ARG, "reader option out of range");
    // the command line's combinations (gtalign.cpp:693-709)
    if (o.split == SPLIT_MODEL && o.ter != TER_EOF)
        return fail(GTB_ERR_ARG, "--split=1 is only compatible with --ter=0");
    if (o.split == SPLIT_CHAIN && o.ter >= TER_END_CHAIN)
        return fail(GTB_ERR_ARG, "--split=2 is only compatible with --ter=0|1");
    for (int i = 0; i < npaths; i++)
        if (!paths[i]) return fail(GTB_ERR_ARG, "null path");
    std::vector<FileResult> res((size_t)npaths);
    int nt = nthreads > 0 ? nthreads : (int)std::thread::hardware_concurrency();
    if (nt < 1) nt = 1;
    if (nt > npaths) nt = npaths > 0 ? npaths : 1;
    std::atomic<int> next{0};
    auto work = [&]() {
        std::string buf;
        for (int i = next++; i < npaths; i = next++) {
            FileResult& r = res[(size_t)i];
            const int fmt = file_format(paths[i], o.infmt);
            if (fmt == 2) {
                std::string tar, ent;
                if (!read_raw(paths[i], tar)) { r.err = std::string("cannot read ") + paths[i]; continue; }
                std::vector<TarEntry> ents;
                if (!tar_entries(tar, ents)) { r.err = std::string(paths[i]) + ": ill-formed tar archive"; continue; }
                for (const TarEntry& e : ents) {
                    const int efmt = file_format(e.name, o.infmt);
                    if (efmt == 2) continue;
                    std::string raw = tar.substr(e.pos, e.size);
                    if (ends_with(e.name, ".gz")) {
                        if (!gunzip(raw, ent)) { r.err = std::string(paths[i]) + ":" + e.name + ": bad gzip data"; break; }
                    } else {
                        ent.swap(raw);
                    }
                    const std::string desc = std::string(paths[i]) + ":" + e.name;
                    if (efmt == 1) parse_cif(desc, ent, o, r);
                    else parse_pdb(desc, ent, o, r);
                    if (!r.err.empty()) break;
                }
                continue;
            }
            FILE* f = std::fopen(paths[i], "rb");
            if (f) {
                std::fseek(f, 0, SEEK_END);
                const long sz = std::ftell(f);
                std::fclose(f);
                if (sz >= 0 && sz < 10) continue;          // too small to list
            }
            // gzip by the name, as the reference decides it; other files as they are
            if (ends_with(paths[i], ".gz")) {
                if (!read_all(paths[i], buf, r.err)) continue;
            } else if (!read_raw(paths[i], buf)) {
                r.err = std::string("cannot open ") + paths[i];
                continue;
            }
            if (fmt == 1) parse_cif(paths[i], buf, o, r);
            else parse_pdb(paths[i], buf, o, r);
        }
    };
    std::vector<std::thread> th;
    for (int t = 1; t < nt; t++) th.emplace_back(work);
    work();
    for (auto& t : th) t.join();
    for (int i = 0; i < npaths; i++)
        if (!res[(size_t)i].err.empty()) return fail(GTB_ERR_ARG, res[(size_t)i].err);
    gtb_structs* b = new gtb_structs();
    size_t ns = 0, np = 0;
    for (auto& r : res) {
        ns += r.strs.size();
        for (auto& s : r.strs) np += s.x.size();
    }
    b->strs.reserve(ns);
    b->len.reserve(ns); b->dist.reserve(ns); b->type.reserve(ns);
    b->x.reserve(np); b->y.reserve(np); b->z.reserve(np);
    b->insch.reserve(np); b->resnum.reserve(np); b->rsd.reserve(np);
    for (auto& r : res)
        for (auto& s : r.strs) {
            b->len.push_back((int)s.x.size());
            b->dist.push_back((unsigned)b->x.size());
            b->type.push_back(s.moltype);
            b->x.insert(b->x.end(), s.x.begin(), s.x.end());
            b->y.insert(b->y.end(), s.y.begin(), s.y.end());
            b->z.insert(b->z.end(), s.z.begin(), s.z.end());
            b->insch.insert(b->insch.end(), s.insch.begin(), s.insch.end());
            b->resnum.insert(b->resnum.end(), s.resnum.begin(), s.resnum.end());
            b->rsd.insert(b->rsd.end(), s.rsd.begin(), s.rsd.end());
            Structure meta;
            meta.desc = s.desc;
            meta.moltype = s.moltype;
            b->strs.push_back(std::move(meta));
            s.clear();
        }
    b->ss.assign(b->x.size(), 0);
    *out = b;
    return GTB_OK;
}

extern "C" gtb_status gtb_structs_size(const gtb_structs* b, int* nstr, long long* npos) {
    if (!b) return GTB_ERR_ARG;
    if (nstr) *nstr = (int)b->len.size();
    if (npos) *npos = (long long)b->x.size();
    return GTB_OK;
}

extern "C" gtb_status gtb_structs_fields(gtb_structs* b, char** pmbeg, char** pmend) {
    if (!b || !pmbeg || !pmend) return GTB_ERR_ARG;
    auto set = [&](int f, void* p, size_t bytes) {
        pmbeg[f] = (char*)p;
        pmend[f] = (char*)p + bytes;
    };
    const size_t n = b->len.size(), N = b->x.size();
    set(GTB_FLD_LEN, b->len.data(), n * sizeof(int));
    set(GTB_FLD_DIST, b->dist.data(), n * sizeof(unsigned));
    set(GTB_FLD_TYPE, b->type.data(), n * sizeof(int));
    set(GTB_FLD_X, b->x.data(), N * sizeof(float));
    set(GTB_FLD_Y, b->y.data(), N * sizeof(float));
    set(GTB_FLD_Z, b->z.data(), N * sizeof(float));
    set(GTB_FLD_INSCHORD, b->insch.data(), N * sizeof(int));
    set(GTB_FLD_RESNUM, b->resnum.data(), N * sizeof(int));
    set(GTB_FLD_RSD, b->rsd.data(), N);
    set(GTB_FLD_SS, b->ss.data(), N);
    return GTB_OK;
}

extern "C" const char* gtb_structs_description(const gtb_structs* b, int i) {
    if (!b || i < 0 || (size_t)i >= b->strs.size()) return nullptr;
    return b->strs[(size_t)i].desc.c_str();
}

extern "C" void gtb_structs_free(gtb_structs* b) { delete b; }
