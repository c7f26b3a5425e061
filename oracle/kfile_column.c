/* Test infrastructure: reads a k file ("(a,b,c)\t<k>\n" rows, the reference
 * programs' output format) from a path (a FIFO works) and writes its k column
 * as one unsigned byte per row to <out>, so that two k files of billions of
 * rows can be compared row by row without holding their text. Exit code 1 on
 * a malformed row or k > 255. */
#include <stdio.h>
#include <stdlib.h>

int main(int argc, char **argv)
{
	if (argc < 3)
	{
		fprintf(stderr, "usage: %s <k file> <k column out>\n", argv[0]);
		return 1;
	}
	FILE *in = fopen(argv[1], "rb"), *out = fopen(argv[2], "wb");
	if (!in || !out)
	{
		fprintf(stderr, "cannot open input or output\n");
		return 1;
	}
	static char buf[1 << 22];
	static unsigned char kout[1 << 22];
	size_t nk = 0, rows = 0;
	int state = 0; /* 0: before the tab, 1: in k */
	unsigned k = 0;
	size_t got;
	while ((got = fread(buf, 1, sizeof buf, in)) > 0)
	{
		for (size_t i = 0; i < got; ++i)
		{
			const char ch = buf[i];
			if (state == 0)
			{
				if (ch == '\t')
				{
					state = 1;
					k = 0;
				}
			}
			else if (ch >= '0' && ch <= '9')
				k = 10 * k + (unsigned)(ch - '0');
			else if (ch == '\n')
			{
				if (k > 255)
				{
					fprintf(stderr, "row %zu: k %u does not fit a byte\n", rows, k);
					return 1;
				}
				kout[nk++] = (unsigned char)k;
				++rows;
				state = 0;
				if (nk == sizeof kout)
				{
					fwrite(kout, 1, nk, out);
					nk = 0;
				}
			}
			else
			{
				fprintf(stderr, "row %zu: unexpected byte %d in k\n", rows, ch);
				return 1;
			}
		}
	}
	fwrite(kout, 1, nk, out);
	fclose(in);
	if (fclose(out) != 0)
		return 1;
	printf("%zu\n", rows);
	return 0;
}
