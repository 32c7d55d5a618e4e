// Entry point for running the reference's own main() (compiled from its main.cpp
// with `main` renamed to capaz_ref_main) unmodified.  Test infrastructure only.
int capaz_ref_main(int argc, char* argv[]);
int main(int argc, char* argv[]) { return capaz_ref_main(argc, argv); }
