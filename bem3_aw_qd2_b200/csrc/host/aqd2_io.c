/* Input files, printing, .dat files and memory of the AQD2 object.
 *
 * Behaviour follows the reference's bem3_aw_qd2.c and aw_pw.c:
 *   read_aqd2            bem3_aw_qd2.c:3-34 (5 or 12 command-line arguments)
 *   read_data_apw        aw_pw.c:3-82       plane-wave file
 *   periodicity file     bem3_aw_qd2.c:424-455
 *   medium file          bem3_aw_qd2.c:468-519
 *   gmsh 2.2 mesh        bem3_aw_qd2.c:531-828: two records per element (main
 *                        and sub domain side, physical tag 99 = open region 0);
 *                        an element whose sub domain is 0 is flipped so that
 *                        domain 0 is always its main domain
 *   dat_write/dat_read   bem3_aw_qd2.c:185-381, byte layout kept
 * Errors print a message and exit, as in the reference.
 */
#include "aqd2_internal.h"

void *aqd2_calloc(size_t n, size_t sz, const char *what)
{
  void *p = calloc(n ? n : 1, sz);
  if (!p) {
    printf("memory allocation error! %s. Exit..\n", what);
    exit(1);
  }
  return p;
}

static void die(const char *file, const char *what)
{
  printf("%s: failed to read %s. exit...\n", file, what);
  exit(1);
}

static void skip_line(FILE *fp, const char *file)
{
  char buf[256];
  if (!fgets(buf, sizeof(buf), fp)) die(file, "a comment line");
}

static double rd(FILE *fp, const char *file, const char *what)
{
  double v;
  if (fscanf(fp, "%lf", &v) != 1) die(file, what);
  return v;
}

static int ri(FILE *fp, const char *file, const char *what)
{
  int v;
  if (fscanf(fp, "%d", &v) != 1) die(file, what);
  return v;
}

void read_data_apw(char *fname, Apw *pw)
{
  FILE *fp = fopen(fname, "rt");
  if (!fp) {
    printf("failed to read %s. no beams defined. Exit...\n", fname);
    exit(1);
  }
  skip_line(fp, fname);
  skip_line(fp, fname);
  pw->rho0 = rd(fp, fname, "rho0");
  pw->c0 = rd(fp, fname, "c0");
  pw->f = rd(fp, fname, "f");
  if (fscanf(fp, "\n") != 0) die(fname, "line end");
  skip_line(fp, fname);
  double re = rd(fp, fname, "real(p)"), im = rd(fp, fname, "imag(p)");
  pw->p = re + I * im;
  for (int i = 0; i < 3; i++) pw->tv[i] = rd(fp, fname, "translation vector");
  pw->theta = rd(fp, fname, "theta");
  pw->psi = rd(fp, fname, "psi");
  fclose(fp);
}

void print_data_apw(Apw *pw)
{
  printf("-- planewave --\n");
  printf("medium density                   [kg/m^3] : %15.14g\n", pw->rho0);
  printf("speed of sound in the medium        [m/s] : %15.14g\n", pw->c0);
  printf("frequency                            [Hz] : %15.14g\n", pw->f);
  printf("sound pressure amplitude             [Pa] :%7.6g+%7.6gI\n", creal(pw->p), cimag(pw->p));
  printf("x-component of translation vector     [m] : %15.14g\n", pw->tv[0]);
  printf("y-component of translation vector     [m] : %15.14g\n", pw->tv[1]);
  printf("z-component of translation vector     [m] : %15.14g\n", pw->tv[2]);
  printf("rotation parameter theta            [rad] : %15.14g\n", pw->theta);
  printf("rotation parameter psi              [rad] : %15.14g\n", pw->psi);
  printf("-- additional information --\n");
  double I0 = 0.5 * creal(pw->p * conj(pw->p)) / (pw->rho0 * pw->c0);
  printf("wavelength                            [m] : %15.14g\n", pw->c0 / pw->f);
  printf("absolute value of sound intensity [W/m^2] : %15.14g\n", I0);
  printf("x-component of sound intensity    [W/m^2] : %15.14g\n", I0 * sin(pw->theta) * cos(pw->psi));
  printf("y-component of sound intensity    [W/m^2] : %15.14g\n", I0 * sin(pw->theta) * sin(pw->psi));
  printf("z-component of sound intensity    [W/m^2] : %15.14g\n", I0 * cos(pw->theta));
  printf("\n");
}

static void read_periodicity(const char *fn, AQD2 *qd)
{
  FILE *fp = fopen(fn, "rt");
  if (!fp) { printf("Can not open the '%s' file. Exit...\n", fn); exit(1); }
  strncpy(qd->ped_fn, fn, sizeof(qd->ped_fn) - 1);
  skip_line(fp, fn);
  skip_line(fp, fn);
  qd->bd.ps = ri(fp, fn, "ps");
  qd->bd.qd.vd1[0] = rd(fp, fn, "vd1");
  qd->bd.qd.vd1[1] = rd(fp, fn, "vd1");
  qd->bd.qd.vd2[0] = rd(fp, fn, "vd2");
  qd->bd.qd.vd2[1] = rd(fp, fn, "vd2");
  fclose(fp);
}

static void read_medium(const char *fn, AQD2 *qd)
{
  FILE *fp = fopen(fn, "rt");
  if (!fp) { printf("Can not open the '%s' file. Exit...\n", fn); exit(1); }
  strncpy(qd->med_fn, fn, sizeof(qd->med_fn) - 1);
  skip_line(fp, fn);
  skip_line(fp, fn);
  qd->MN = ri(fp, fn, "MN");
  if (fscanf(fp, "\n") != 0) die(fn, "line end");
  int n = qd->MN + 1;
  qd->rho0 = (double *)aqd2_calloc(n, sizeof(double), "rho0");
  qd->c0 = (double *)aqd2_calloc(n, sizeof(double), "c0");
  qd->k0 = (double *)aqd2_calloc(n, sizeof(double), "k0");
  qd->K0 = (double *)aqd2_calloc(n, sizeof(double), "K0");
  qd->k1 = (double complex *)aqd2_calloc(n, sizeof(double complex), "k1");
  qd->k2 = (double complex *)aqd2_calloc(n, sizeof(double complex), "k2");
  skip_line(fp, fn);
  for (int i = 1; i <= qd->MN; i++) {
    qd->rho0[i] = rd(fp, fn, "rho0");
    qd->c0[i] = rd(fp, fn, "c0");
  }
  fclose(fp);
}

void aqd2_malloc_node(BOUD *bd)
{
  bd->rn = (double **)aqd2_calloc(bd->Nn + 1, sizeof(double *), "rn");
  for (int i = 0; i <= bd->Nn; i++) bd->rn[i] = (double *)aqd2_calloc(3, sizeof(double), "rn[i]");
}

void aqd2_malloc_elem(BOUD *bd)
{
  int Ne = bd->Ne;
  bd->ed = (int **)aqd2_calloc(Ne + 1, sizeof(int *), "ed");
  bd->eni = (int **)aqd2_calloc(Ne + 1, sizeof(int *), "eni");
  bd->md = (int *)aqd2_calloc(Ne + 1, sizeof(int), "md");
  bd->sd = (int *)aqd2_calloc(Ne + 1, sizeof(int), "sd");
  bd->gd = (int *)aqd2_calloc(Ne + 1, sizeof(int), "gd");
  bd->cr = (double ***)aqd2_calloc(Ne + 1, sizeof(double **), "cr");
  bd->cw = (double ***)aqd2_calloc(Ne + 1, sizeof(double **), "cw");
  bd->ren = (double ***)aqd2_calloc(Ne + 1, sizeof(double **), "ren");
  bd->wen = (double ***)aqd2_calloc(Ne + 1, sizeof(double **), "wen");
  bd->Pi = (double complex **)aqd2_calloc(Ne + 1, sizeof(double complex *), "Pi");
  bd->dPi = (double complex **)aqd2_calloc(Ne + 1, sizeof(double complex *), "dPi");
  for (int i = 0; i <= Ne; i++) {
    bd->ed[i] = (int *)aqd2_calloc(4, sizeof(int), "ed[i]");
    bd->eni[i] = (int *)aqd2_calloc(4, sizeof(int), "eni[i]");
    bd->cr[i] = (double **)aqd2_calloc(3, sizeof(double *), "cr[i]");
    bd->cw[i] = (double **)aqd2_calloc(3, sizeof(double *), "cw[i]");
    for (int j = 0; j < 3; j++) {
      bd->cr[i][j] = (double *)aqd2_calloc(4, sizeof(double), "cr[i][j]");
      bd->cw[i][j] = (double *)aqd2_calloc(3, sizeof(double), "cw[i][j]");
    }
    bd->ren[i] = (double **)aqd2_calloc(4, sizeof(double *), "ren[i]");
    bd->wen[i] = (double **)aqd2_calloc(4, sizeof(double *), "wen[i]");
    for (int j = 0; j < 4; j++) {
      bd->ren[i][j] = (double *)aqd2_calloc(3, sizeof(double), "ren[i][j]");
      bd->wen[i][j] = (double *)aqd2_calloc(3, sizeof(double), "wen[i][j]");
    }
    bd->Pi[i] = (double complex *)aqd2_calloc(4, sizeof(double complex), "Pi[i]");
    bd->dPi[i] = (double complex *)aqd2_calloc(4, sizeof(double complex), "dPi[i]");
  }
}

/* physical tag of a gmsh record -> domain id (99 is the open region 0) */
static int tag_domain(int tag, const AQD2 *qd)
{
  if (tag == OPENDID) tag = 0;
  if (tag > qd->MN || tag < 0) {
    printf("domain id %d is not defined medium data. check domain and medium data. exit..\n", tag);
    exit(1);
  }
  return tag;
}

static void read_mesh(const char *fn, AQD2 *qd)
{
  FILE *fp = fopen(fn, "rt");
  if (!fp) { printf("Can not open the '%s' file. Exit...\n", fn); exit(1); }
  strncpy(qd->msh_fn, fn, sizeof(qd->msh_fn) - 1);
  skip_line(fp, fn);  /* $MeshFormat */
  double ver = rd(fp, fn, "version");
  if (ver < 2.2) { printf("This program supports mesh file version 2.2 later. Reading file version is %g. Exit...\n", ver); exit(1); }
  if (ri(fp, fn, "format") != 0) { printf("This program supports 'ASCII' data format mesh file. Exit...\n"); exit(1); }
  if (ri(fp, fn, "precision") != 8) { printf("This program supports double precision mesh data. Exit...\n"); exit(1); }
  if (fscanf(fp, "\n") != 0) die(fn, "line end");
  skip_line(fp, fn);  /* $EndMeshFormat */
  skip_line(fp, fn);  /* $Nodes */
  BOUD *bd = &qd->bd;
  bd->Nn = ri(fp, fn, "node count");
  aqd2_malloc_node(bd);
  for (int i = 1; i <= bd->Nn; i++) {
    int id = ri(fp, fn, "node id");
    if (id != i) printf("bad id %d\n", id);
    for (int d = 0; d < 3; d++) bd->rn[i][d] = rd(fp, fn, "node coordinate");
  }
  if (fscanf(fp, "\n") != 0) die(fn, "line end");
  skip_line(fp, fn);  /* $EndNodes */
  skip_line(fp, fn);  /* $Elements */
  bd->Ne = ri(fp, fn, "element count") / 2;
  aqd2_malloc_elem(bd);
  int nc = 0;
  for (int i = 1; i <= bd->Ne; i++) {
    int nid[4], nid2[4];
    /* first record: main-domain side */
    if (ri(fp, fn, "element id") != 2 * i - 1) { printf("bad id. Exit...\n"); exit(1); }
    int et = ri(fp, fn, "element type");
    if (et != ELT3 && et != ELT4) { printf("bad element type. element type must be %d or %d. Exit...\n", ELT3, ELT4); exit(1); }
    int nt = ri(fp, fn, "tag count");
    for (int j = 0; j < nt; j++) {
      int tg = ri(fp, fn, "tag");
      if (j == 0) bd->md[i] = tag_domain(tg, qd);
      else if (j == 1) bd->gd[i] = tg;
    }
    int nv = et == ELT3 ? 3 : 4;
    for (int j = 0; j < nv; j++) nid[j] = ri(fp, fn, "node");
    for (int j = 0; j < 4; j++) bd->ed[i][j] = j < nv ? nid[j] : 0;
    for (int j = 0; j < 4; j++) bd->eni[i][j] = j < nv ? nc++ : -1;
    /* second record: the same element seen from the sub domain (reversed order) */
    if (ri(fp, fn, "element id") != 2 * i) { printf("bad id. Exit...\n"); exit(1); }
    int et2 = ri(fp, fn, "element type");
    if (et2 != ELT3 && et2 != ELT4) { printf("bad element type. element type must be %d or %d. Exit...\n", ELT3, ELT4); exit(1); }
    nt = ri(fp, fn, "tag count");
    for (int j = 0; j < nt; j++) {
      int tg = ri(fp, fn, "tag");
      if (j == 0) bd->sd[i] = tag_domain(tg, qd);
    }
    for (int j = 0; j < nv; j++) nid2[j] = ri(fp, fn, "node");
    int ok = nid2[0] == nid[0];
    for (int j = 1; j < nv; j++) ok = ok && nid2[j] == nid[nv - j];
    if (!ok) { printf("node id miss matched. check element id %d. Exit...\n", 2 * i); exit(1); }
    if (bd->sd[i] == 0) {  /* make the open region the main domain */
      bd->sd[i] = bd->md[i];
      bd->md[i] = 0;
      int a = nv == 3 ? 1 : 1, b = nv == 3 ? 2 : 3;
      int tmp = bd->ed[i][a];
      bd->ed[i][a] = bd->ed[i][b];
      bd->ed[i][b] = tmp;
    }
  }
  fclose(fp);
  bd->NN = nc;
}

void read_aqd2(int argc, char **argv, AQD2 *qd)
{
  if (argc != 6 && argc != 13) {
    printf("This program needs command line arguments as follows.\n");
    printf("%s plane_wave_datafile_name periodicity_datafile_name medium_datafile_name mesh_datafile_name output_datafile_name\n", argv[0]);
    printf("[rv_x rv_y rv_z theta tr_x tr_y tr_z](optional)\n");
    printf("rv : vector defining rotation axis, theta : rotation angle ( using Rodrigues' rotation formula ), tr : translation vector\n");
    exit(0);
  }
  memset(qd, 0, sizeof(*qd));
  read_data_apw(argv[1], &qd->pw);
  read_periodicity(argv[2], qd);
  read_medium(argv[3], qd);
  read_mesh(argv[4], qd);
  if (argc == 13) {
    for (int i = 0; i < 3; i++) qd->rv[i] = atof(argv[6 + i]);
    qd->th = atof(argv[9]);
    for (int i = 0; i < 3; i++) qd->tv[i] = atof(argv[10 + i]);
  } else {
    qd->rv[0] = 1.0; qd->rv[1] = 0.0; qd->rv[2] = 0.0;
    qd->th = 0.0;
    qd->tv[0] = qd->tv[1] = qd->tv[2] = 0.0;
  }
}

void print_aqd2(AQD2 *qd)
{
  print_data_apw(&qd->pw);
  printf("--- periodicity data ---\n");
  printf("periodicity data file name = %s\n", qd->ped_fn);
  printf("periodicity setting        = %10d\n", qd->bd.ps);
  printf("lattice constant d1        = (% 7g,% 7g)\n", qd->bd.qd.vd1[0], qd->bd.qd.vd1[1]);
  printf("lattice constant d2        = (% 7g,% 7g)\n", qd->bd.qd.vd2[0], qd->bd.qd.vd2[1]);
  printf("\n");
  printf("--- medium data ---\n");
  printf("medium data file name      = %s\n", qd->med_fn);
  for (int i = 1; i <= qd->MN; i++) {
    printf("domain id %2d rho0 [kg/m^3] =%8.6g\n", i, qd->rho0[i]);
    printf("             c0      [m/s] =%8.6g\n", qd->c0[i]);
  }
  printf("\n");
  printf("--- mesh data ---\n");
  printf("mesh data file name        = %s\n", qd->msh_fn);
  printf("node number                = %8d\n", qd->bd.Nn);
  printf("defined element number     = %8d\n", qd->bd.Ne * 2);
  printf("\n");
  double atv = sqrt(qd->tv[0] * qd->tv[0] + qd->tv[1] * qd->tv[1] + qd->tv[2] * qd->tv[2]);
  if (qd->th != 0.0 || atv != 0.0) {
    printf("-- rotation and translation settings --\n");
    if (qd->th != 0.0) {
      printf("vector defining rotation axis :(% 8.7g,% 8.7g,% 8.7g)\n", qd->rv[0], qd->rv[1], qd->rv[2]);
      printf("rotation angle           [rad]: %8.7g\n", qd->th);
    }
    if (atv != 0.0) printf("translation vector            :(%8.7g,%8.7g,%8.7g)\n", qd->tv[0], qd->tv[1], qd->tv[2]);
  }
  printf("\n");
}

void aqd2_malloc_sub_domain(AQD2 *qd)
{
  int n = qd->MN + 1;
  int *Nc = (int *)aqd2_calloc(n, sizeof(int), "Nc");
  for (int i = 1; i <= qd->bd.Ne; i++) {
    Nc[qd->bd.md[i]]++;
    Nc[qd->bd.sd[i]]++;
  }
  qd->bd.sb = (SUBD *)aqd2_calloc(n, sizeof(SUBD), "sb");
  for (int d = 0; d < n; d++) {
    SUBD *s = &qd->bd.sb[d];
    s->Ne = Nc[d];
    s->sid = (int *)aqd2_calloc(Nc[d] + 1, sizeof(int), "sid");
    s->P = (double complex **)aqd2_calloc(Nc[d] + 1, sizeof(double complex *), "P");
    s->dP = (double complex **)aqd2_calloc(Nc[d] + 1, sizeof(double complex *), "dP");
    s->pv = (double complex ***)aqd2_calloc(Nc[d] + 1, sizeof(double complex **), "pv");
    s->dpv = (double complex ***)aqd2_calloc(Nc[d] + 1, sizeof(double complex **), "dpv");
    for (int j = 0; j <= Nc[d]; j++) {
      s->P[j] = (double complex *)aqd2_calloc(4, sizeof(double complex), "P[j]");
      s->dP[j] = (double complex *)aqd2_calloc(4, sizeof(double complex), "dP[j]");
      s->pv[j] = (double complex **)aqd2_calloc(4, sizeof(double complex *), "pv[j]");
      s->dpv[j] = (double complex **)aqd2_calloc(4, sizeof(double complex *), "dpv[j]");
      for (int k = 0; k < 4; k++) {
        s->pv[j][k] = (double complex *)aqd2_calloc(3, sizeof(double complex), "pv[j][k]");
        s->dpv[j][k] = (double complex *)aqd2_calloc(3, sizeof(double complex), "dpv[j][k]");
      }
    }
  }
  free(Nc);
}

void finalize_aqd2(AQD2 *qd)
{
  aqd2_release_device(qd);
  BOUD *bd = &qd->bd;
  if (bd->sb) {
    for (int d = 0; d <= qd->MN; d++) {
      SUBD *s = &bd->sb[d];
      for (int j = 0; j <= s->Ne; j++) {
        free(s->P[j]);
        free(s->dP[j]);
        for (int k = 0; k < 4; k++) { free(s->pv[j][k]); free(s->dpv[j][k]); }
        free(s->pv[j]);
        free(s->dpv[j]);
      }
      free(s->sid); free(s->P); free(s->dP); free(s->pv); free(s->dpv);
    }
    free(bd->sb);
    bd->sb = NULL;
  }
  if (bd->ed) {
    for (int i = 0; i <= bd->Ne; i++) {
      free(bd->ed[i]); free(bd->eni[i]);
      for (int j = 0; j < 3; j++) { free(bd->cr[i][j]); free(bd->cw[i][j]); }
      free(bd->cr[i]); free(bd->cw[i]);
      for (int j = 0; j < 4; j++) { free(bd->ren[i][j]); free(bd->wen[i][j]); }
      free(bd->ren[i]); free(bd->wen[i]); free(bd->Pi[i]); free(bd->dPi[i]);
    }
    free(bd->ed); free(bd->eni); free(bd->md); free(bd->sd); free(bd->gd);
    free(bd->cr); free(bd->cw); free(bd->ren); free(bd->wen); free(bd->Pi); free(bd->dPi);
    bd->ed = NULL;
    bd->Ne = 0;
  }
  if (bd->rn) {
    for (int i = 0; i <= bd->Nn; i++) free(bd->rn[i]);
    free(bd->rn);
    bd->rn = NULL;
    bd->Nn = 0;
  }
  free(qd->rho0); free(qd->c0); free(qd->k0); free(qd->K0); free(qd->k1); free(qd->k2);
  qd->rho0 = qd->c0 = qd->k0 = qd->K0 = NULL;
  qd->k1 = qd->k2 = NULL;
}

/* ------------------------------------------------------------------ .dat */
static void wr(const void *p, size_t sz, size_t n, FILE *fp, const char *fn)
{
  if (fwrite(p, sz, n, fp) != n) { printf("failed to write the %s file. exit...\n", fn); exit(1); }
}

static void rdb(void *p, size_t sz, size_t n, FILE *fp, const char *what)
{
  if (fread(p, sz, n, fp) != n) { printf("bem3_aw_qd2 dat_read_aqd2(), failed to read the %s. exit...\n", what); exit(1); }
}

void dat_write_aqd2(char *fname, AQD2 *qd)
{
  FILE *fp = fopen(fname, "wb");
  if (!fp) { printf("dat_write_aqd2(), Failed to create the %s file.\n", fname); exit(1); }
  BOUD *bd = &qd->bd;
  int n = qd->MN + 1;
  wr(qd, sizeof(AQD2), 1, fp, fname);
  wr(qd->rho0, sizeof(double), n, fp, fname);
  wr(qd->c0, sizeof(double), n, fp, fname);
  wr(qd->k0, sizeof(double), n, fp, fname);
  wr(qd->K0, sizeof(double), n, fp, fname);
  wr(qd->k1, sizeof(double complex), n, fp, fname);
  wr(qd->k2, sizeof(double complex), n, fp, fname);
  wr(&qd->pw, sizeof(Apw), 1, fp, fname);
  for (int i = 0; i <= bd->Nn; i++) wr(bd->rn[i], sizeof(double), 3, fp, fname);
  for (int i = 0; i <= bd->Ne; i++) wr(bd->ed[i], sizeof(int), 4, fp, fname);
  for (int i = 0; i <= bd->Ne; i++) wr(bd->eni[i], sizeof(int), 4, fp, fname);
  wr(bd->md, sizeof(int), bd->Ne + 1, fp, fname);
  wr(bd->sd, sizeof(int), bd->Ne + 1, fp, fname);
  wr(bd->gd, sizeof(int), bd->Ne + 1, fp, fname);
  for (int i = 0; i <= bd->Ne; i++) for (int j = 0; j < 4; j++) wr(bd->ren[i][j], sizeof(double), 3, fp, fname);
  for (int i = 0; i <= bd->Ne; i++) for (int j = 0; j < 4; j++) wr(bd->wen[i][j], sizeof(double), 3, fp, fname);
  for (int i = 0; i <= bd->Ne; i++) wr(bd->Pi[i], sizeof(double complex), 4, fp, fname);
  for (int i = 0; i <= bd->Ne; i++) wr(bd->dPi[i], sizeof(double complex), 4, fp, fname);
  for (int d = 0; d < n; d++) {
    SUBD *s = &bd->sb[d];
    wr(&s->Ne, sizeof(int), 1, fp, fname);
    wr(s->sid, sizeof(int), s->Ne + 1, fp, fname);
    for (int i = 0; i <= s->Ne; i++) wr(s->P[i], sizeof(double complex), 4, fp, fname);
    for (int i = 0; i <= s->Ne; i++) wr(s->dP[i], sizeof(double complex), 4, fp, fname);
    for (int i = 0; i <= s->Ne; i++) for (int j = 0; j < 4; j++) wr(s->pv[i][j], sizeof(double complex), 3, fp, fname);
    for (int i = 0; i <= s->Ne; i++) for (int j = 0; j < 4; j++) wr(s->dpv[i][j], sizeof(double complex), 3, fp, fname);
  }
  fclose(fp);
}

void dat_read_aqd2(char *fname, AQD2 *qd)
{
  FILE *fp = fopen(fname, "rb");
  if (!fp) { printf("dat_read_aqd2(), Failed to open the %s file.\n", fname); exit(1); }
  rdb(qd, sizeof(AQD2), 1, fp, "qd");
  BOUD *bd = &qd->bd;
  int n = qd->MN + 1;
  qd->rho0 = (double *)aqd2_calloc(n, sizeof(double), "rho0");
  qd->c0 = (double *)aqd2_calloc(n, sizeof(double), "c0");
  qd->k0 = (double *)aqd2_calloc(n, sizeof(double), "k0");
  qd->K0 = (double *)aqd2_calloc(n, sizeof(double), "K0");
  qd->k1 = (double complex *)aqd2_calloc(n, sizeof(double complex), "k1");
  qd->k2 = (double complex *)aqd2_calloc(n, sizeof(double complex), "k2");
  rdb(qd->rho0, sizeof(double), n, fp, "rho0");
  rdb(qd->c0, sizeof(double), n, fp, "c0");
  rdb(qd->k0, sizeof(double), n, fp, "k0");
  rdb(qd->K0, sizeof(double), n, fp, "K0");
  rdb(qd->k1, sizeof(double complex), n, fp, "k1");
  rdb(qd->k2, sizeof(double complex), n, fp, "k2");
  rdb(&qd->pw, sizeof(Apw), 1, fp, "pw");
  aqd2_malloc_node(bd);
  aqd2_malloc_elem(bd);
  for (int i = 0; i <= bd->Nn; i++) rdb(bd->rn[i], sizeof(double), 3, fp, "rn");
  for (int i = 0; i <= bd->Ne; i++) rdb(bd->ed[i], sizeof(int), 4, fp, "ed");
  for (int i = 0; i <= bd->Ne; i++) rdb(bd->eni[i], sizeof(int), 4, fp, "eni");
  rdb(bd->md, sizeof(int), bd->Ne + 1, fp, "md");
  rdb(bd->sd, sizeof(int), bd->Ne + 1, fp, "sd");
  rdb(bd->gd, sizeof(int), bd->Ne + 1, fp, "gd");
  for (int i = 0; i <= bd->Ne; i++) for (int j = 0; j < 4; j++) rdb(bd->ren[i][j], sizeof(double), 3, fp, "ren");
  for (int i = 0; i <= bd->Ne; i++) for (int j = 0; j < 4; j++) rdb(bd->wen[i][j], sizeof(double), 3, fp, "wen");
  for (int i = 0; i <= bd->Ne; i++) rdb(bd->Pi[i], sizeof(double complex), 4, fp, "Pi");
  for (int i = 0; i <= bd->Ne; i++) rdb(bd->dPi[i], sizeof(double complex), 4, fp, "dPi");
  aqd2_init_elem_const(bd);
  aqd2_malloc_sub_domain(qd);
  for (int d = 0; d < n; d++) {
    SUBD *s = &bd->sb[d];
    int tmp;
    rdb(&tmp, sizeof(int), 1, fp, "Ne");
    rdb(s->sid, sizeof(int), s->Ne + 1, fp, "sid");
    for (int i = 0; i <= s->Ne; i++) rdb(s->P[i], sizeof(double complex), 4, fp, "P");
    for (int i = 0; i <= s->Ne; i++) rdb(s->dP[i], sizeof(double complex), 4, fp, "dP");
    for (int i = 0; i <= s->Ne; i++) for (int j = 0; j < 4; j++) rdb(s->pv[i][j], sizeof(double complex), 3, fp, "pv");
    for (int i = 0; i <= s->Ne; i++) for (int j = 0; j < 4; j++) rdb(s->dpv[i][j], sizeof(double complex), 3, fp, "dpv");
  }
  fclose(fp);
}
