/*
 * poa_oracle_cli.c - command-line front end of the CPU restatement
 * (TEST INFRASTRUCTURE). Mirrors the subset of minipoa's CLI that the hot
 * path covers (src/main.cpp:14-35): -M -X -O -E -b -f -B -r {0,1,2}.
 * With -d FILE it also writes one record per read:
 *   A <read index> <score> <path length>
 *   <from>,<base>,<aligned_id> ...
 * the same format oracle/ref_harness.cpp writes for the reference.
 */
#include "poa_oracle.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef struct { char *name, *comment, *seq; int len; } rec;

static rec *read_fasta(const char *path, int *n) {
    FILE *fp = fopen(path, "rb");
    if (!fp) { perror(path); exit(2); }
    fseek(fp, 0, SEEK_END);
    long sz = ftell(fp);
    fseek(fp, 0, SEEK_SET);
    char *buf = (char *)malloc((size_t)sz + 1);
    if (fread(buf, 1, (size_t)sz, fp) != (size_t)sz) { perror("read"); exit(2); }
    buf[sz] = 0;
    fclose(fp);
    int cap = 16, cnt = 0;
    rec *r = (rec *)malloc(sizeof(rec) * cap);
    char *s = buf;
    while (*s) {
        if (*s != '>' && *s != '@') { s++; continue; }
        char fq = *s == '@';
        s++;
        char *eol = strchr(s, '\n');
        if (!eol) eol = s + strlen(s);
        char *hdr_end = eol;
        if (hdr_end > s && hdr_end[-1] == '\r') hdr_end--;
        char *sp = s;
        while (sp < hdr_end && *sp != ' ' && *sp != '\t') sp++;
        if (cnt == cap) { cap *= 2; r = (rec *)realloc(r, sizeof(rec) * cap); }
        r[cnt].name = strndup(s, (size_t)(sp - s));
        r[cnt].comment = sp < hdr_end ? strndup(sp + 1, (size_t)(hdr_end - sp - 1)) : strdup("");
        s = *eol ? eol + 1 : eol;
        size_t scap = 1024, sl = 0;
        char *sq = (char *)malloc(scap);
        while (*s && *s != '>' && !(fq && *s == '+')) {
            if (*s == '@' && !fq) break;
            if (*s != '\n' && *s != '\r') {
                if (sl + 1 >= scap) { scap *= 2; sq = (char *)realloc(sq, scap); }
                sq[sl++] = *s;
            }
            s++;
        }
        if (fq && *s == '+') { /* skip the quality block of the same length */
            char *e2 = strchr(s, '\n'); s = e2 ? e2 + 1 : s + strlen(s);
            size_t ql = 0;
            while (*s && ql < sl) { if (*s != '\n' && *s != '\r') ql++; s++; }
        }
        sq[sl] = 0;
        r[cnt].seq = sq; r[cnt].len = (int)sl;
        cnt++;
    }
    free(buf);
    *n = cnt;
    return r;
}

int main(int argc, char **argv) {
    po_params p;
    po_params_default(&p);
    int mode = 0;
    const char *in = NULL, *dump = NULL;
    for (int a = 1; a < argc; a++) {
        const char *o = argv[a];
        if (!strcmp(o, "-B")) p.ab_band = 1;
        else if (!strcmp(o, "-M") && a + 1 < argc) p.match = atoi(argv[++a]);
        else if (!strcmp(o, "-X") && a + 1 < argc) p.mismatch = atoi(argv[++a]);
        else if (!strcmp(o, "-O") && a + 1 < argc) p.gap_open1 = atoi(argv[++a]);
        else if (!strcmp(o, "-E") && a + 1 < argc) p.gap_ext1 = atoi(argv[++a]);
        else if (!strcmp(o, "-b") && a + 1 < argc) p.b = atoi(argv[++a]);
        else if (!strcmp(o, "-f") && a + 1 < argc) p.f = atoi(argv[++a]);
        else if (!strcmp(o, "-r") && a + 1 < argc) mode = atoi(argv[++a]);
        else if (!strncmp(o, "-r", 2) && o[2]) mode = atoi(o + 2);
        else if (!strcmp(o, "-d") && a + 1 < argc) dump = argv[++a];
        else in = o;
    }
    if (!in) { fprintf(stderr, "usage: poa_oracle in.fa [-B] [-r 0|1|2] [-M -X -O -E -b -f] [-d dump]\n"); return 2; }
    po_params_normalize(&p);
    int n;
    rec *r = read_fasta(in, &n);
    FILE *df = dump ? fopen(dump, "w") : NULL;
    po_graph *g = po_graph_new();
    for (int i = 0; i < n; i++) {
        uint8_t *q = (uint8_t *)malloc((size_t)r[i].len + 1);
        for (int j = 0; j < r[i].len; j++) q[j] = po_nt4((uint8_t)r[i].seq[j]);
        po_res *path; int plen, sc = 0;
        int st = po_alignment(g, &p, q, r[i].len, &path, &plen, &sc);
        free(q);
        if (st == PO_BAND_ESCAPE) return 0; /* the reference exit(0)s here */
        if (st != PO_OK) { fprintf(stderr, " backtrack error\n"); return 1; }
        if (df && po_graph_nnodes(g) > 2) {
            fprintf(df, "A %d %d %d\n", i, sc, plen);
            for (int k = 0; k < plen; k++)
                fprintf(df, "%d,%d,%d%c", path[k].from, path[k].base, path[k].aligned_id, k + 1 == plen ? '\n' : ' ');
            if (plen == 0) fputc('\n', df);
        }
        po_add_path(g, i, path, plen, 1);
        free(path);
        po_topsort(g, &p, i + 1 == n);
    }
    if (df) fclose(df);
    if (mode == 0) {
        int len;
        char *c = po_consensus(g, &len);
        printf(">consensus sequence\n%s\n", c);
        free(c);
    } else if (mode == 2) {
        int *lens = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
        const char **names = (const char **)malloc(sizeof(char *) * (size_t)(n > 0 ? n : 1));
        for (int i = 0; i < n; i++) { lens[i] = r[i].len; names[i] = r[i].name; }
        char *t = po_gfa(g, n, lens, names);
        fputs(t, stdout);
        free(t);
        free(lens);
        free((void *)names);
    } else {
        int nc;
        char *rows = po_msa(g, n, &nc);
        for (int i = 0; i < n; i++) {
            if (r[i].name[0] == 0) printf(">%d\n", i + 1);
            else printf(">%s %s\n", r[i].name, r[i].comment);
            fwrite(rows + (size_t)i * nc, 1, (size_t)nc, stdout);
            fputc('\n', stdout);
        }
        free(rows);
    }
    po_graph_free(g);
    return 0;
}
