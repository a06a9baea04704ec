# Prints one brace-balanced block of a reference source file, for oracle/_ref host builds
# (test infrastructure; the output goes to oracle/_ref/gen only, never into the repository).
#   awk -v anchor='PROFILE("Gen Tids")' -v start='KRR_DEVICE_LAMBDA(const int tid) {' \
#       -f extract_block.awk integrator.cpp
# After the first line containing `anchor`, the first line containing `start` opens the block;
# lines are printed until the braces opened there close. A trailing comma after the closing
# brace (a lambda passed as an argument) is dropped. With anchor empty, `start` alone is used.
BEGIN { state = (anchor == "") ? 1 : 0; depth = 0 }
{ sub(/\r$/, "") }
state == 0 && index($0, anchor) { state = 1 }
state == 1 && index($0, start) { state = 2 }
state == 2 {
    line = $0
    opened = gsub(/\{/, "{", line)
    closed = gsub(/\}/, "}", line)
    depth += opened - closed
    if (depth == 0) {
        sub(/\}[ \t]*,[ \t]*$/, "}", line)
        print line
        found = 1
        exit
    }
    print line
}
END { if (!found) { print "extract_block: block not found" > "/dev/stderr"; exit 1 } }
